"""Device resolution with the reference's priority rule
(atom3d/core/device_utils.py:12-57): explicit device argument, then the
device of the first tensor given, then the default."""

from __future__ import annotations

from typing import Optional, Union

import torch


def resolve_device(*tensors: Optional[torch.Tensor], device: Optional[Union[str, torch.device]] = None,
                   default: str = "cuda") -> torch.device:
    if device is not None:
        return device if isinstance(device, torch.device) else torch.device(device)
    for t in tensors:
        if isinstance(t, torch.Tensor):
            return t.device
    if default == "cuda" and not torch.cuda.is_available():
        return torch.device("cpu")
    return torch.device(default)
