from .bound import LearnedBound, train_for_mesh

__all__ = ["LearnedBound", "train_for_mesh"]
