"""Benchmark of the closest-point (UDF) hot path on B200.

Workload: icosphere level 8 (655,362 vertices, 1,310,720 triangles)
radially displaced by 16 seeded sinusoids (amplitude 0.05 each), 16,777,216
queries: half area-weighted surface samples + N(0, 0.02), half uniform in
the mesh box scaled by 1.2.  One step = one closest-point pass over all
queries (distance, face id, closest point) through the C ABI.

  value  : queries/s with inputs resident in HBM (device-timed, CUDA events)
  e2e    : queries/s through MeshBVH.udf with pinned host buffers, H2D of
           the queries and D2H of the results inside the timed region;
           consecutive steps overlap as in a serving loop (the next step's
           input copy and this step's result copy on two copy streams beside
           the traversal); serial_value: the same with no overlap
  roofline.achieved : algorithmic bytes of the traversal kernel per launch
           (32 B of I/O + 24 B per node box + 36 B per triangle test of the
           plain method on the reference's binary tree, per query) / its
           average CUDA-event duration
  cpu_baseline : the CPU brute-force port of the reference's closest-point
           maths on a bounded query sample, all host threads

Multi-GPU (torchrun): replicas only (weak scaling); each rank runs the full
workload on its own GPU, value = total queries / max-over-ranks time.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
"""

from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np
import torch
import torch.distributed as dist

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)

METRIC = "UDF Mqueries/s (plain traversal, 1.31M-triangle mesh, 16M queries)"
# DRAM read + write of one udf_task_kernel launch per query, measured by an
# ncu capture of a 4,194,304-query launch on this mesh (1.471 GB); traffic
# scales with the query count (the tree stays in L2)
DRAM_BYTES_PER_QUERY = 1.471343e9 / 4194304
TRAFFIC_SOURCE = "ncu dram__bytes_read.sum + dram__bytes_write.sum, 4,194,304-query capture scaled per query"
UNIT = "Mqueries/s"
WORKLOAD = "udf_large: icosphere L8 (1,310,720 tris) + 16 sinusoids, 16,777,216 mixed queries"

# Per-query algorithmic traversal counts of the plain method on the
# reference's binary SAH tree (counted once by the oracle's instrumented
# restatement of bvh_udf_kernel over the reference build_bvh output for this
# mesh, on a 16,384-query sample of this distribution; see
# tests/golden/make_traversal_counts.py).  Bytes per unit: node 24 B,
# triangle 36 B, compulsory 32 B per query.
COUNTS_FILE = os.path.join(HERE, "tests", "golden", "udf_large_counts.json")


def load_counts():
    try:
        with open(COUNTS_FILE) as f:
            return json.load(f)
    except OSError:
        return None


def peaks():
    p = os.path.join(HERE, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi sampling during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.idx = gpu_index
        self.proc = None
        self.path = None

    def __enter__(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.idx), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        rows = []
        try:
            with open(self.path) as f:
                for line in f:
                    parts = [x.strip() for x in line.split(",")]
                    if len(parts) >= 9:
                        rows.append(parts)
        except OSError:
            pass
        finally:
            try:
                os.unlink(self.path)
            except OSError:
                pass
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"], "samples": 0}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


def flush_l2(buf):
    buf.add_(1.0)


def setup_dist(gpus):
    """One process per GPU: (rank, world size, local rank).  NCCL on a GPU box;
    gloo where CUDA is absent (the CPU tests of the replica bookkeeping)."""
    if gpus > 1 or "RANK" in os.environ:
        backend = "nccl" if torch.cuda.is_available() else "gloo"
        dist.init_process_group(backend=backend, timeout=__import__("datetime").timedelta(seconds=300))
        rank = dist.get_rank()
        local = int(os.environ.get("LOCAL_RANK", rank))
        return rank, dist.get_world_size(), local
    return 0, 1, 0


def barrier(world):
    if world > 1:
        dist.barrier()


def max_over_ranks(x, world, dev):
    if world == 1:
        return x
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_throughput(units_per_rank, world, max_ms):
    """Whole-job rate of N independent replicas: all ranks' units over the
    slowest rank's time (millions of units per second)."""
    return units_per_rank * world / (max_ms * 1e-3) / 1e6


def cpu_baseline(v, f, q, budget_s=15.0):
    """Brute-force CPU port of the reference's closest-point maths (oracle),
    on a bounded prefix of the query set, all host threads."""
    from oracle import orc

    orc.build()
    n = 64
    t = 0.0
    while True:
        t0 = time.perf_counter()
        orc.ref_udf_bruteforce(v.numpy(), f.numpy(), q[:n].numpy())
        t = time.perf_counter() - t0
        if t > budget_s / 4 or n >= 8192:
            break
        n *= 2
    return {"value": n / t / 1e6, "unit": UNIT, "cores": orc.threads(), "kind": "port",
            "sample": f"{n} of the 16,777,216 queries (brute force over all 1,310,720 triangles)"}


def fp64_check(v, f, q, dist_d, fid_d, n_sample=1024):
    """Error of the device results against the oracle's FP64 brute force on a
    stratified sample (half surface-band, half box queries): max distance
    error (absolute and over the box diagonal) and face ids exact or tied."""
    from oracle import orc

    n = q.shape[0]
    g = np.random.default_rng(2024)
    h = n_sample // 2
    pick = np.sort(np.concatenate([g.choice(n // 2, h, replace=False), n // 2 + g.choice(n - n // 2, h, replace=False)]))
    pt = torch.from_numpy(pick).to(dist_d.device)
    d = dist_d[pt].double().cpu().numpy()
    fid = fid_d[pt].cpu().numpy()
    qs = q[pick].numpy()
    t0 = time.perf_counter()
    d64, f64, _ = orc.udf_exact(v.numpy(), f.numpy(), qs)
    diag = float((v.double().max(0).values - v.double().min(0).values).norm())
    err = float(np.abs(d - d64).max())
    dm = orc.tri_dist(v.numpy(), f.numpy(), qs, fid)
    tie = np.abs(dm - d64) <= 1e-6 * diag
    return {"sample": int(pick.shape[0]), "max_abs_err": err, "max_err_over_diag": err / diag,
            "face_ids_exact": float((fid == f64).mean()), "face_ids_exact_or_tie": float(((fid == f64) | tie).mean()),
            "oracle": "FP64 brute force over all triangles", "oracle_s": time.perf_counter() - t0}


def reference_gpu_bar(steps=3):
    """The reference's own CUDA kernels (compiled from its sources into
    oracle/_ref with its flags) on this GPU: its host SAH build, bvh_udf on
    the 16,777,216-query workload, and octree_traverse 4 -> 10 plus
    sparse_flood_fill at 1024^3 (the 327,680-triangle sphere) driven by the
    restated host glue.  Wall-clock with synchronisation (the reference's
    flood fill runs on the legacy default stream with a host loop)."""
    from oracle import ref_gpu

    if not torch.cuda.is_available():
        return {"unavailable": "no CUDA device"}
    if not ref_gpu.available():
        return {"unavailable": "oracle/_ref not built (oracle/build_ref.py needs the reference checkout)"}
    from atom3d_b200 import synthetic

    dev = torch.device("cuda", 0)
    out = {"build": "reference sources, -O3 --use_fast_math, sm_100a (oracle/build_ref.py)"}

    def wall(fn, k):
        fn()
        torch.cuda.synchronize()
        ts = []
        for _ in range(k):
            t0 = time.perf_counter()
            fn()
            torch.cuda.synchronize()
            ts.append(time.perf_counter() - t0)
        return statistics.median(ts) * 1e3

    v, f, q = synthetic.udf_large()
    t0 = time.perf_counter()
    rb = ref_gpu.RefBVH(v.to(dev), f.to(dev))
    torch.cuda.synchronize()
    build_s = time.perf_counter() - t0
    qd = q.to(dev)
    ms = wall(lambda: rb.udf(qd), steps)
    out["udf"] = {"queries": int(q.shape[0]), "ms": ms, "Mqueries_per_s": q.shape[0] / ms / 1e3,
                  "host_sah_build_s": build_s}
    del qd, rb
    v2, f2 = synthetic.octree_mesh()
    rb2 = ref_gpu.RefBVH(v2.to(dev), f2.to(dev))
    bounds = torch.tensor([[-1.5] * 3, [1.5] * 3])
    oct_ms = wall(lambda: ref_gpu.octree_traverse(rb2, bounds, 4, 10), steps)
    dam = ref_gpu.octree_traverse(rb2, bounds, 4, 10)

    def flood():
        water, dry, coll, tdam, _, _ = ref_gpu.flood_fill_3d_sparse(dam, 1024, padding=10, connectivity=26)
        ref_gpu.dam_neighborhood_signs(tdam, water, dry, 1024, 1)

    flood_ms = wall(flood, max(1, steps - 1))
    out["octree_flood_1024"] = {"octree_ms": oct_ms, "flood_fill_ms": flood_ms, "candidates": int(dam.shape[0])}
    return out


def run_reference(args):
    rank, world, local = setup_dist(args.gpus)
    if rank != 0:
        if world > 1:
            dist.destroy_process_group()
        return
    from atom3d_b200 import synthetic

    v, f, q = synthetic.udf_large()
    base = cpu_baseline(v, f, q, budget_s=20.0)
    steps = []
    from oracle import orc

    n = int(base["sample"].split()[0])
    for _ in range(args.warmup + args.steps):
        t0 = time.perf_counter()
        orc.ref_udf_bruteforce(v.numpy(), f.numpy(), q[:n].numpy())
        steps.append(time.perf_counter() - t0)
    t = statistics.mean(steps[args.warmup:])
    val = n / t / 1e6
    base["value"] = val
    line = {"impl": "reference", "metric": METRIC, "value": val, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": t * 1e3, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": WORKLOAD, "sample_queries": n},
            "cpu_baseline": base, "e2e": {"value": val, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    try:
        line["reference_gpu"] = reference_gpu_bar()
    except Exception as e:  # the reference's GPU bar is a reported extra
        line["reference_gpu"] = {"unavailable": f"{type(e).__name__}: {e}"}
    dmc_golden = os.path.join(HERE, "tests", "golden", "dmc512.npz")
    if os.path.exists(dmc_golden):
        g = np.load(dmc_golden)
        line["reference_cpu_dmc_512"] = {
            "forward_s": float(g["ref_cpu_s"][0]), "backward_s": float(g["ref_cpu_s"][1]),
            "cubes": int(g["n_cubes"]), "where": "build container, 8 threads (tests/golden/make_dmc512_golden.py); "
            "the reference's SparseDiffDMC is Python and is not on the GPU machine"}
    print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--queries", type=int, default=16 * 1024 * 1024)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-extra", action="store_true", help="skip every measurement besides the main UDF line")
    ap.add_argument("--skip", default="", help="comma-separated extra sections to skip: learned,dmc,octree,rays,batch")
    ap.add_argument("--section", default="", choices=["", "dmc", "octree", "rays", "batch", "build", "learned"],
                    help="run one extra section alone on cuda:0 and print its JSON (for profiling)")
    ap.add_argument("--level", type=int, default=10, help="octree section: finest level (10 = 1024^3)")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    if args.impl == "reference":
        return run_reference(args)
    if args.section:
        return run_section(args)

    rank, world, local = setup_dist(args.gpus)
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    from atom3d_b200 import MeshBVH, _lib, synthetic

    v, f, q = synthetic.udf_large(n_queries=args.queries)
    n = q.shape[0]
    mesh = MeshBVH(v.to(dev), f.to(dev))
    qd = q.to(dev)
    bvh = mesh._bvh
    flags = _lib.A3D_UDF_SORT_QUERIES | int(os.environ.get("ATOM3D_B200_UDF_FLAGS", "0"))
    dist_o = torch.empty(n, device=dev)
    fid_o = torch.empty(n, dtype=torch.int32, device=dev)
    cp_o = torch.empty(n, 3, device=dev)
    ws = _lib.workspace(_lib.lib().a3d_udf_workspace_bytes(n, flags), dev)
    import ctypes

    view = bvh.view
    stream = torch.cuda.current_stream(dev)

    def step(stats=None):
        _lib.call("a3d_udf", ctypes.byref(view), qd.data_ptr(), n, dist_o.data_ptr(), fid_o.data_ptr(),
                  cp_o.data_ptr(), None, None, None, _lib.ptr(stats), flags, ws.data_ptr(), ws.numel(),
                  stream.cuda_stream)

    # traversal statistics of our tree (one untimed pass)
    st = torch.zeros(4, dtype=torch.int64, device=dev)
    step(st)
    torch.cuda.synchronize()
    our_nodes, our_tris, reruns, rounds = (int(x) for x in st[:4].cpu())

    for _ in range(args.warmup):
        step()
    barrier(world)
    torch.cuda.synchronize()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        ev0.record(stream)
        for _ in range(args.steps):
            step()
        ev1.record(stream)
        torch.cuda.synchronize()
    barrier(world)
    ms = ev0.elapsed_time(ev1) / args.steps
    ms = max_over_ranks(ms, world, dev)
    clocks = clk.summary()

    # dominant kernel duration: time the traversal launch alone (queries
    # pre-sorted by one untimed call; same stream, CUDA events)
    kernel_ms = time_traversal_kernel(bvh, qd, dist_o, fid_o, cp_o, ws, flags, stream, args.steps)

    # end to end through the public API, pinned host buffers
    qh = q.pin_memory()
    dh = torch.empty(n, pin_memory=True)
    fh = torch.empty(n, dtype=torch.int32, pin_memory=True)
    ch = torch.empty(n, 3, pin_memory=True)

    def e2e_step():
        qq = qh.to(dev, non_blocking=True)
        r = mesh.udf(qq, return_closest=True, return_face_ids=True)
        dh.copy_(r.distances, non_blocking=True)
        fh.copy_(r.face_ids, non_blocking=True)
        ch.copy_(r.closest_points, non_blocking=True)

    for _ in range(2):
        e2e_step()
    barrier(world)
    torch.cuda.synchronize()
    ev0.record(stream)
    for _ in range(args.steps):
        e2e_step()
    ev1.record(stream)
    torch.cuda.synchronize()
    e2e_serial_ms = max_over_ranks(ev0.elapsed_time(ev1) / args.steps, world, dev)

    # the same steps as a serving loop runs them: step i+1's queries are
    # copied in on one copy stream and step i's results copied out on
    # another while the traversal of the next step runs; every step still
    # copies its own queries in and its own results out inside the timed
    # region (two device input buffers; each result set is read back before
    # its memory is reused)
    copy_in, copy_out = torch.cuda.Stream(dev), torch.cuda.Stream(dev)
    qbuf = [torch.empty_like(qd) for _ in range(2)]
    in_ready = [torch.cuda.Event() for _ in range(2)]
    buf_free = [torch.cuda.Event() for _ in range(2)]

    def e2e_pipelined(k):
        with torch.cuda.stream(copy_in):
            qbuf[0].copy_(qh, non_blocking=True)
            in_ready[0].record(copy_in)
        for i in range(k):
            b = i % 2
            stream.wait_event(in_ready[b])
            r = mesh.udf(qbuf[b], return_closest=True, return_face_ids=True)
            buf_free[b].record(stream)
            if i + 1 < k:
                with torch.cuda.stream(copy_in):
                    if i > 0:  # buffer 1 - b was last read by step i - 1
                        copy_in.wait_event(buf_free[1 - b])
                    qbuf[1 - b].copy_(qh, non_blocking=True)
                    in_ready[1 - b].record(copy_in)
            with torch.cuda.stream(copy_out):
                copy_out.wait_event(buf_free[b])
                for t in (r.distances, r.face_ids, r.closest_points):
                    t.record_stream(copy_out)
                dh.copy_(r.distances, non_blocking=True)
                fh.copy_(r.face_ids, non_blocking=True)
                ch.copy_(r.closest_points, non_blocking=True)
        stream.wait_stream(copy_out)

    e2e_pipelined(2)
    barrier(world)
    torch.cuda.synchronize()
    ev0.record(stream)
    e2e_pipelined(args.steps)
    ev1.record(stream)
    torch.cuda.synchronize()
    e2e_ms = max_over_ranks(ev0.elapsed_time(ev1) / args.steps, world, dev)

    peak, peak_kind = peaks()
    counts = load_counts()
    roof = None
    if counts is not None:
        per_q = 32.0 + 24.0 * counts["nodes_per_query"] + 36.0 * counts["tris_per_query"]
        achieved = per_q * n / (kernel_ms * 1e-3) / 1e9
        roof = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                "traffic": DRAM_BYTES_PER_QUERY * n, "traffic_source": TRAFFIC_SOURCE, "peak_kind": peak_kind,
                "bytes_per_query": per_q, "kernel": "udf_task_kernel", "kernel_ms": kernel_ms}
        # the tree (nodes + triangles, ~91 MB) stays in L2: the same bytes
        # against the L2 read bandwidth measured on this GPU
        l2 = l2_read_peak(dev)
        roof["l2"] = {"peak": l2, "unit": "GB/s", "frac": achieved / l2,
                      "how": "a3d_read_probe: 48 MiB buffer read 40 times through L2 (16-B ld.global.cg), "
                             "CUDA events, best of 5"}
    line = {
        "metric": METRIC, "value": replica_throughput(n, world, ms), "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32", "data": "synthetic",
        "config": {"workload": WORKLOAD, "queries_per_gpu": n, "triangles": int(f.shape[0]),
                   "parallelism": f"replicas{world}", "l2": "inputs larger than L2 (192 MB queries, 512 MB outputs)"},
        "e2e": {"value": replica_throughput(n, world, e2e_ms), "unit": UNIT, "h2d_bytes_per_step": n * 12,
                "d2h_bytes_per_step": n * (4 + 4 + 12),
                "how": "MeshBVH.udf per step from pinned host queries to pinned host results; the next step's "
                       "input copy and this step's result copy on two copy streams beside the traversal",
                "serial_value": replica_throughput(n, world, e2e_serial_ms)},
        "roofline": roof,
        "gpu_launches": args.steps * launches_per_udf(),
        "clocks": clocks,
        "traversal": {"nodes_per_query": our_nodes / n, "tris_per_query": our_tris / n, "reruns": reruns,
                      "warp_rounds_per_query": rounds / n},
    }
    skip = set(x for x in args.skip.split(",") if x)
    if not args.no_extra:
        cpu = rank == 0 and not args.no_cpu_baseline
        if "learned" not in skip:
            line["learned"] = bench_learned(dev, v, f, mesh, qd, max(3, args.steps // 2))
        if "dmc" not in skip:
            line["dmc"] = bench_dmc(dev, max(2, args.steps // 2), 2, cpu=cpu)
        if "octree" not in skip:
            line["octree_flood"] = bench_octree_flood(dev, max(2, args.steps // 2), 3)
        if "rays" not in skip:
            line["rays"] = bench_rays(dev, mesh, v, max(3, args.steps // 2))
        if "batch" not in skip:
            line["batch"] = bench_batch(dev, 2, 1, cpu=cpu)
        if "build" not in skip:
            line["build"] = bench_build(dev, max(3, args.steps // 2))
    if rank == 0 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(v, f, q)
        step()
        torch.cuda.synchronize()
        line["fp64_check"] = fp64_check(v, f, q, dist_o, fid_o)
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()


def run_section(args):
    """One extra section alone (its own workload and timing), for profiling."""
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    steps = max(2, args.steps)
    if args.section == "dmc":
        out = bench_dmc(dev, steps, args.warmup, cpu=False)
    elif args.section == "octree":
        out = bench_octree_flood(dev, steps, args.warmup, max_level=args.level)
    elif args.section == "batch":
        out = bench_batch(dev, 2, 1, cpu=False)
    elif args.section == "build":
        out = bench_build(dev, steps)
    elif args.section == "learned":
        from atom3d_b200 import MeshBVH, synthetic

        v, f, q = synthetic.udf_large(n_queries=args.queries)
        out = bench_learned(dev, v, f, MeshBVH(v.to(dev), f.to(dev)), q.to(dev), steps)
    else:
        from atom3d_b200 import MeshBVH, synthetic

        v, f, _ = synthetic.udf_large(n_queries=2)
        out = bench_rays(dev, MeshBVH(v.to(dev), f.to(dev)), v, steps)
    print(json.dumps({"section": args.section, **out}), flush=True)


def bench_build(dev, steps):
    """GPU BVH build of the 1,310,720-triangle mesh (Morton codes, radix sort,
    radix tree, SAH refinement, refit with the collapse costs, collapse,
    layout), device-timed.  Algorithmic bytes per triangle: 60 (Morton) +
    24 per 8-bit radix pass x 8 passes + 80 (emission and refit)."""
    from atom3d_b200 import MeshBVH, synthetic

    v, f, _ = synthetic.udf_large(n_queries=2)
    vd, fd = v.to(dev), f.to(dev)
    MeshBVH(vd, fd)
    ms = _time_ms(lambda: MeshBVH(vd, fd), steps)
    nf = int(f.shape[0])
    peak, kind = peaks()
    byts = (60 + 24 * 8 + 80) * nf
    gbs = byts / (ms * 1e-3) / 1e9
    return {"metric": "BVH build ms (1,310,720 triangles)", "value": ms, "unit": "ms", "triangles": nf,
            "roofline": {"bound": "hbm", "achieved": gbs, "peak": peak, "unit": "GB/s", "frac": gbs / peak,
                         "peak_kind": kind, "bytes": "332 B per triangle (60 Morton + 8 x 24 radix + 80 refit)",
                         "note": "whole build call incl. host read of its node count; latency-bound"}}


def _time_ms(fn, steps, warmup=2):
    for _ in range(warmup):
        fn()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(steps):
        fn()
    e1.record()
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / steps


def bench_learned(dev, v, f, mesh, qd, steps):
    """Learned-bound UDF vs plain on the 16M-query workload: the bound MLP is
    trained on 4,194,304 plain-method samples of the same distribution
    (other seed) with the hand-written BF16 kernels; every variant returns
    identical distances and face ids (checked here)."""
    from atom3d_b200 import _lib, synthetic
    from atom3d_b200.learned import train_for_mesh

    n = qd.shape[0]
    g = torch.Generator().manual_seed(77)
    train = synthetic.mixed_queries(v, f, 1 << 22, g)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    lb = train_for_mesh(mesh, train, epochs=8, coverage=0.99, tune=True, log_space=True)
    torch.cuda.synchronize()
    train_s = time.perf_counter() - t0
    bvh = mesh._bvh
    ref = bvh.query(qd)
    bound = lb(qd)
    exact = torch.nextafter(ref[0], torch.full_like(ref[0], float("inf"))) * (1 + 1e-6)
    infer_ms = _time_ms(lambda: lb(qd, out=bound), steps)
    NR, BS = _lib.A3D_UDF_NO_REUSE, _lib.A3D_UDF_BOUND_SEEDS
    variants = {
        "plain": (None, 0),
        "plain_no_neighbour_seed": (None, NR),
        "learned_cap": (bound, 0),
        "learned_seeds": (bound, NR | BS),
        "exact_bound_cap": (exact, 0),
        "exact_bound_seeds": (exact, NR | BS),
    }
    out = {"metric": "UDF Mqueries/s, learned bound vs plain (same 16M queries)", "unit": UNIT,
           "train_s": train_s, "train_samples": 1 << 22, "margin": lb.margin, "scale": lb.scale,
           "coverage": lb.coverage, "log_space": lb.log_space,
           "infer_ms": infer_ms, "infer_tflops": 82176 * n / (infer_ms * 1e-3) / 1e12,
           "bound_covers": float((ref[0] <= bound).float().mean())}
    for name, (b, flags) in variants.items():
        st = torch.zeros(4, dtype=torch.int64, device=dev)
        r = bvh.query(qd, bound=b, seeding=flags, stats=st)
        same = bool(torch.equal(r[0], ref[0]) and torch.equal(r[1], ref[1]))
        nodes, tris, reruns, _ = (int(x) for x in st.cpu())
        ms = _time_ms(lambda: bvh.query(qd, bound=b, seeding=flags), steps)
        if name.startswith("learned"):
            ms += infer_ms  # the bound's inference is part of the learned path
        # per-query node visits and triangle tests (a query whose bound
        # excluded every triangle counts both of its passes)
        out[name] = {"ms": ms, "mqs": n / ms / 1e3, "identical": same, "nodes_per_query": nodes / n,
                     "tris_per_query": tris / n, "deep_stack_reruns": reruns}
    out["speedup_learned_vs_plain"] = out["plain"]["ms"] / min(out["learned_cap"]["ms"], out["learned_seeds"]["ms"])
    out["speedup_exact_bound_vs_plain"] = out["plain"]["ms"] / min(out["exact_bound_cap"]["ms"],
                                                                     out["exact_bound_seeds"]["ms"])
    return out


def bench_rays(dev, mesh, v, steps):
    """Ray queries on the 1.31M-triangle mesh: nearest hit for 16,777,216 rays
    (origins uniform in the 1.2x box, uniform directions), all hits for
    1,048,576 of them, and the ray-parity SDF (8 directions) for 1,048,576
    points."""
    g = torch.Generator().manual_seed(31)
    n = 1 << 24
    lo, hi = v.min(0).values, v.max(0).values
    c, h = (lo + hi) * 0.5, (hi - lo) * 0.6
    o = (c + (torch.rand(n, 3, generator=g) * 2 - 1) * h).float().to(dev)
    d = torch.randn(n, 3, generator=g)
    d = (d / d.norm(dim=1, keepdim=True)).float().to(dev)
    near_ms = _time_ms(lambda: mesh.intersect_ray(o, d), steps)
    r = mesh.intersect_ray(o, d)
    m = 1 << 20
    all_ms = _time_ms(lambda: mesh.intersect_ray(o[:m], d[:m], mode="all"), steps)
    ra = mesh.intersect_ray(o[:m], d[:m], mode="all")
    par_ms = _time_ms(lambda: mesh.sdf(o[:m], mode="parity"), steps)
    return {"metric": "ray queries on the 1.31M-triangle mesh", "unit": "Mrays/s",
            "nearest": {"rays": n, "ms": near_ms, "mrays_s": n / near_ms / 1e3,
                        "hit_fraction": float(r.hit.float().mean())},
            "all_hits": {"rays": m, "ms": all_ms, "mrays_s": m / all_ms / 1e3, "hits": int(ra.t.numel())},
            "parity_sdf": {"points": m, "directions": 8, "ms": par_ms, "mpoints_s": m / par_ms / 1e3},
            "status": mesh.ray_status()}


def launches_per_batch(num_queries, num_meshes):
    """Kernels of one batched build + query (the graph's kernel nodes)."""
    mbits = max(0, int(np.ceil(np.log2(max(num_meshes, 1)))))
    bits = min(21, (64 - mbits) // 3)
    sort_passes = -(-(3 * bits + mbits) // 8)
    build = 3 + 5 * sort_passes + 3 + 64 + 2 + 5 + 3
    chunks = -(-num_queries // (1 << 24))
    qbits = min(10, (32 - mbits) // 3)
    per_chunk = 1 + 5 * (-(-(3 * qbits + mbits) // 8)) + 2
    return build + chunks * per_chunk


def bench_batch(dev, steps, warmup, cpu=True):
    """256 displaced icospheres (levels 3-8, 74.6M triangles) under seeded
    affine maps, 8 queries per triangle (597M); one step = the batched
    build + UDF of all meshes replayed from a captured CUDA graph."""
    from atom3d_b200 import synthetic
    from atom3d_b200.batch import BatchedMeshBVH, offsets

    t0 = time.perf_counter()
    meshes = synthetic.batch_meshes(256, seed=4, device=dev)
    vc = [int(m[0].shape[0]) for m in meshes]
    fc = [int(m[1].shape[0]) for m in meshes]
    qc = [int(m[2].shape[0]) for m in meshes]
    V = torch.cat([m[0] for m in meshes]).contiguous()
    F = torch.cat([m[1] for m in meshes]).int().contiguous()
    Q = torch.cat([m[2] for m in meshes]).contiguous()
    sample_meshes = [(m[0].cpu(), m[1].cpu(), m[2][:: max(1, m[2].shape[0] // 8)][:8].cpu()) for m in meshes]
    del meshes
    torch.cuda.synchronize()
    gen_s = time.perf_counter() - t0
    nq, nf = int(Q.shape[0]), int(F.shape[0])
    bb = BatchedMeshBVH(vertices=V, faces=F, vertex_counts=vc, face_counts=fc)
    qoff = offsets(qc, dev)
    tune = bb.autotune(Q, qoff, sample=1 << 21)
    dist_o = torch.empty(nq, device=dev)
    fid_o = torch.empty(nq, dtype=torch.int32, device=dev)
    cp_o = torch.empty(nq, 3, device=dev)
    st = torch.zeros(4, dtype=torch.int64, device=dev)
    bb.udf_into(Q, qoff, dist_o, fid_o, cp_o, stats=st)
    torch.cuda.synchronize()
    stats = [int(x) for x in st.cpu()]
    build_ms = _time_ms(bb.build, 3, 1)
    query_ms = _time_ms(lambda: bb.udf_into(Q, qoff, dist_o, fid_o, cp_o), 1, 0)
    g = bb.capture(Q, qoff, dist_o, fid_o, cp_o)
    with ClockSampler(dev.index or 0) as clk:
        ms = _time_ms(g.replay, steps, warmup)
    status = bb.query_status()
    bb.check()
    out = {"metric": "batched build + UDF, Mqueries/s (256 meshes, 74.6M tris, 597M queries, CUDA graph)",
           "value": nq / ms / 1e3, "unit": UNIT, "ms_per_step": ms, "steps": steps, "warmup": warmup,
           "meshes": len(fc), "triangles": nf, "queries": nq, "build_ms": build_ms, "query_ms": query_ms,
           "generate_s": gen_s, "autotune": tune, "status": status, "clocks": clk.summary(),
           "gpu_launches": steps * launches_per_batch(nq, len(fc)),
           "traversal": {"nodes_per_query": stats[0] / nq, "tris_per_query": stats[1] / nq, "reruns": stats[2]}}
    # end to end: pinned host mesh + queries in, distances + face ids +
    # closest points out, around the same graph
    try:
        hV, hF, hQ = V.cpu().pin_memory(), F.cpu().pin_memory(), Q.cpu().pin_memory()
        hd = torch.empty(nq, pin_memory=True)
        hf = torch.empty(nq, dtype=torch.int32, pin_memory=True)
        hc = torch.empty(nq, 3, pin_memory=True)

        def e2e():
            bb.vertices.copy_(hV, non_blocking=True)
            bb.faces.copy_(hF, non_blocking=True)
            Q.copy_(hQ, non_blocking=True)
            g.replay()
            hd.copy_(dist_o, non_blocking=True)
            hf.copy_(fid_o, non_blocking=True)
            hc.copy_(cp_o, non_blocking=True)

        e_ms = _time_ms(e2e, 1, 1)
        out["e2e"] = {"value": nq / e_ms / 1e3, "unit": UNIT, "h2d_bytes_per_step": hV.numel() * 4 + hF.numel() * 4
                      + hQ.numel() * 4, "d2h_bytes_per_step": nq * 20}
        del hV, hF, hQ, hd, hf, hc
    except RuntimeError as e:  # pinned host memory is limited on some hosts
        out["e2e"] = {"value": None, "unavailable": str(e)[:200]}
    if cpu:
        from oracle import orc

        orc.build()
        t0 = time.perf_counter()
        done = 0
        for v_, f_, q_ in sample_meshes:
            orc.ref_udf_bruteforce(v_.numpy(), f_.numpy(), q_.numpy())
            done += q_.shape[0]
        t = time.perf_counter() - t0
        out["cpu_baseline"] = {"value": done / t / 1e6, "unit": UNIT, "cores": orc.threads(), "kind": "port",
                               "sample": f"{done} queries, 8 per mesh, brute force over each mesh's triangles"}
    del g
    return out


def bench_dmc(dev, steps, warmup, cpu=True):
    """SparseDiffDMC forward + backward (loss = sum |v|^2, grad w.r.t. sdf) on
    the 32-sphere union sampled at 512^3 (2.2M active cubes)."""
    from atom3d_b200 import SparseDiffDMC, synthetic

    vox, sdf, cidx, _ = synthetic.dmc_spheres(res=512)
    vd, sd, cd = vox.to(dev), sdf.to(dev), cidx.to(dev)
    dmc = SparseDiffDMC(device=str(dev))

    def fwd_bwd():
        s_ = sd.detach().requires_grad_(True)
        o = dmc(vd, s_, cd, 512)
        (o.vertices ** 2).sum().backward()
        return o

    def fwd_only():
        return dmc(vd, sd.detach().requires_grad_(True), cd, 512)

    # steps back to back between two events on the stream (the forward's two
    # host reads of counts stay inside each step); backward = the difference
    o = fwd_bwd()
    # each step is about a millisecond: time at least 20 of them after 5
    # warm-up steps so allocator and clock effects average out
    tot = _time_ms(fwd_bwd, max(20, steps), max(5, warmup))
    fwd = _time_ms(fwd_only, max(20, steps), max(5, warmup))
    n_cubes, n_v, n_f = vox.shape[0], o.vertices.shape[0], o.faces.shape[0]
    peak, kind = peaks()
    alg = 108.0 * n_cubes + 12.0 * n_v + 24.0 * n_f
    out = {"metric": "DMC fwd+bwd ms (32-sphere SDF, 512^3, 2.2M active cubes)", "value": tot, "unit": "ms",
           "higher_is_better": False, "fwd_ms": fwd, "bwd_ms": tot - fwd, "active_cubes": int(n_cubes),
           "vertices": int(n_v), "faces": int(n_f),
           "roofline_fwd": {"bound": "hbm", "achieved": alg / (fwd * 1e-3) / 1e9, "peak": peak, "unit": "GB/s",
                            "frac": alg / (fwd * 1e-3) / 1e9 / peak, "peak_kind": kind,
                            "bytes": "108 B/active cube + 12 B/vertex + 24 B/face"}}
    dmc_eval = SparseDiffDMC(device=str(dev)).eval()
    with torch.no_grad():
        eval_ms = _time_ms(lambda: dmc_eval(vd, sd, cd, 512), steps)
        oe = dmc_eval(vd, sd, cd, 512)
    out["eval_qef"] = {"ms": eval_ms, "vertices": int(oe.vertices.shape[0]), "faces": int(oe.faces.shape[0]),
                       "note": "inference mode: corner gradients + QEF vertices + 2-triangle split, forward only"}
    if cpu:
        from oracle import dmc_oracle, orc

        t0 = time.perf_counter()
        dmc_oracle.forward(vox.numpy(), sdf.numpy(), cidx.numpy(), 512)
        t = time.perf_counter() - t0
        out["cpu_baseline"] = {"value": t * 1e3, "unit": "ms", "cores": orc.threads(), "kind": "port",
                               "sample": "full forward only (numpy restatement of the reference's train mode)"}
    return out


def bench_octree_flood(dev, steps, warmup, max_level=10):
    """octree_traverse (levels 4..max_level, 1024^3 by default) and
    sparse_flood_fill on the 327,680-triangle displaced sphere, bounds
    [-1.5, 1.5]^3."""
    from atom3d_b200 import MeshBVH, OctreeIndexer, sparse_flood_fill, synthetic

    v, f = synthetic.octree_mesh()
    bounds = torch.tensor([[-1.5] * 3, [1.5] * 3], device=dev)
    stream = torch.cuda.current_stream(dev)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    vd, fd = v.to(dev), f.to(dev)
    MeshBVH(vd, fd)  # first build of the process: module load and allocations
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    mesh = MeshBVH(vd, fd)
    torch.cuda.synchronize()
    build_ms = (time.perf_counter() - t0) * 1e3
    oc = OctreeIndexer(max_level=max_level, bounds=bounds, device=dev)
    res_grid = 1 << max_level
    for _ in range(warmup):
        cand = oc.octree_traverse(mesh, min_level=4)
    torch.cuda.synchronize()
    e0.record(stream)
    for _ in range(steps):
        cand = oc.octree_traverse(mesh, min_level=4)
    e1.record(stream)
    torch.cuda.synchronize()
    oct_ms = e0.elapsed_time(e1) / steps
    # each call returns ~4.8 GB of label coordinates: the previous result is
    # released before the next call, so the timed calls reuse its memory
    # instead of timing fresh device allocations
    out = None
    for _ in range(max(2, warmup - 1)):
        out = None
        out = sparse_flood_fill(mesh, res_grid, min_level=4, bounds=bounds, verbose=False)
    torch.cuda.synchronize()
    e0.record(stream)
    for _ in range(steps):
        out = None
        out = sparse_flood_fill(mesh, res_grid, min_level=4, bounds=bounds, verbose=False)
    e1.record(stream)
    torch.cuda.synchronize()
    ff_ms = e0.elapsed_time(e1) / steps
    labels = {k: int(t.shape[0]) for k, t in out.items()}
    # reference-layout traffic per visited voxel (water + collision): the
    # BFS's 26 hash probes of 8 B, a 4 B label write and two 4 B frontier
    # entries; the timed call includes its own octree descent
    visited = labels["water_ijk"] + labels["tide_ijk"]
    peak, kind = peaks()
    gbs = 220.0 * visited / (ff_ms * 1e-3) / 1e9
    res = {"metric": f"octree SAT 4->{max_level} + sparse flood fill at {res_grid}^3 (327,680 tris)", "unit": "ms",
           "bvh_build_ms": build_ms, "octree_ms": oct_ms, "sparse_flood_fill_ms": ff_ms,
           "candidate_voxels": int(cand.shape[0]), "labels": labels,
           "roofline_flood": {"bound": "hbm", "achieved": gbs, "peak": peak, "unit": "GB/s", "frac": gbs / peak,
                              "peak_kind": kind, "visited_voxels": visited,
                              "bytes": "220 B per visited voxel (water + collision), the reference BFS's traffic; "
                                       "time of the whole sparse_flood_fill call incl. its octree descent"}}
    res["dual_graph"] = bench_dual(dev, oc, out, steps)
    res["aabb_pairs"] = bench_pairs(dev, mesh, oc, cand, steps)
    return res


def bench_dual(dev, oc, labels, steps):
    """construct_surface_dual_graph of the flood fill's dam + tide +
    dry-adjacent cells at 1024^3, and the three dam wet masks.  Algorithmic
    bytes: 12 B read per listed cell; 12 B cell + 64 B cube_idx + 48 B
    adj_idx written per active cell, 24 B ijk + 12 B world per vertex."""
    from atom3d_b200.apps import (construct_surface_dual_graph, get_dam_wet_corners, get_dam_wet_edges,
                                  get_dam_wet_faces)

    dam, tide, dry = labels["dam_ijk"], labels["tide_ijk"], labels["dry_adjacent_ijk"]
    g_ms = _time_ms(lambda: construct_surface_dual_graph(dam, tide, dry, oc), steps)
    w, vijk, ci, adj, cells = construct_surface_dual_graph(dam, tide, dry, oc)
    n_in = dam.shape[0] + tide.shape[0] + dry.shape[0]
    alg = 12.0 * n_in + 124.0 * cells.shape[0] + 36.0 * vijk.shape[0]
    peak, kind = peaks()
    R = 1 << int(oc.max_level)
    wet_ms = _time_ms(lambda: (get_dam_wet_faces(dam, tide, R), get_dam_wet_edges(dam, tide, R),
                               get_dam_wet_corners(dam, tide, R)), steps)
    return {"ms": g_ms, "active_cells": int(cells.shape[0]), "vertices": int(vijk.shape[0]),
            "listed_cells": int(n_in),
            "roofline": {"bound": "hbm", "achieved": alg / (g_ms * 1e-3) / 1e9, "peak": peak, "unit": "GB/s",
                         "frac": alg / (g_ms * 1e-3) / 1e9 / peak, "peak_kind": kind,
                         "bytes": "12 B/listed cell + 124 B/active cell + 36 B/vertex (whole call, host syncs included)"},
            "wet_masks_ms": wet_ms, "dam_cells": int(dam.shape[0])}


def bench_pairs(dev, mesh, oc, cand, steps):
    """MeshBVH.intersect_aabb on the level-10 octree candidates of the
    327,680-triangle mesh (mode 1: SAT pairs; mode 3: clipped polygons), and
    the reference demo's workload (80-face icosphere at 512^3, mode 3)."""
    from atom3d_b200 import MeshBVH, OctreeIndexer, synthetic

    mn, mx = oc.cube_aabb_level(cand, int(oc.max_level))
    out = {"boxes": int(mn.shape[0])}
    for mode in (1, 3):
        ms = _time_ms(lambda: mesh.intersect_aabb(mn, mx, mode=mode), steps)
        r = mesh.intersect_aabb(mn, mx, mode=mode)
        out[f"mode{mode}"] = {"ms": ms, "pairs": int(r.aabb_ids.numel()), "mpairs_s": r.aabb_ids.numel() / ms / 1e3}
    v, f = synthetic.icosphere(1)
    ico = MeshBVH(v.to(dev), f.to(dev))
    oc9 = OctreeIndexer(max_level=9, bounds=ico.get_bounds(), device=dev)
    c9 = oc9.octree_traverse(ico)
    a, b = oc9.cube_aabb_level(c9, 9)
    ms = _time_ms(lambda: ico.intersect_aabb(a, b, mode=3), steps)
    r = ico.intersect_aabb(a, b, mode=3)
    out["demo_icosphere_512"] = {"boxes": int(a.shape[0]), "ms": ms, "polygons": int(r.poly_counts.numel()),
                                 "reference_demo_polygons": 1172044,
                                 "poly_counts_range": [int(r.poly_counts.min()), int(r.poly_counts.max())]}
    return out


def l2_read_peak(dev, mib=48, passes=40, reps=5):
    """Read bandwidth of a buffer that stays in L2 (GB/s): a3d_read_probe
    streams it `passes` times; best of `reps` CUDA-event timings."""
    import ctypes

    from atom3d_b200 import _lib

    fn = _lib.lib().a3d_read_probe
    fn.restype = ctypes.c_int
    fn.argtypes = [ctypes.c_void_p, ctypes.c_int64, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p]
    buf = torch.ones(mib << 20, dtype=torch.uint8, device=dev)
    sink = torch.zeros(1, dtype=torch.int32, device=dev)
    stream = torch.cuda.current_stream(dev)
    nbytes = buf.numel()

    def run():
        _lib.check("a3d_read_probe", fn(buf.data_ptr(), nbytes, passes, sink.data_ptr(), stream.cuda_stream))

    run()
    best = float("inf")
    for _ in range(reps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        run()
        e1.record(stream)
        torch.cuda.synchronize(dev)
        best = min(best, e0.elapsed_time(e1))
    return nbytes * passes / (best * 1e-3) / 1e9


def launches_per_udf():
    # query Morton keys (1) + 4 radix passes x (upsweep, 3 scan kernels,
    # downsweep) + traversal + re-run kernel
    return 1 + 4 * 5 + 2


def time_traversal_kernel(bvh, qd, dist_o, fid_o, cp_o, ws, flags, stream, steps):
    """Average duration of the traversal launch itself: the same call on
    pre-sorted queries with A3D_UDF_ASSUME_SORTED, so only the traversal
    kernel (plus its empty re-run launch) is inside the events."""
    import ctypes

    from atom3d_b200 import _lib, synthetic  # noqa: F401

    n = qd.shape[0]
    # Morton order of the queries (same key as the library) via one sorted call
    lo = torch.tensor(bvh.lo, device=qd.device)
    hi = torch.tensor(bvh.hi, device=qd.device)
    emax = float((hi - lo).max())
    c = (lo + hi) * 0.5 - emax
    key = ((qd - c) * (1023.0 / (2 * emax))).clamp(0, 1023).to(torch.int64)
    code = torch.zeros(n, dtype=torch.int64, device=qd.device)
    for b in range(10):
        for a in range(3):
            code |= ((key[:, a] >> b) & 1) << (3 * b + a)
    order = torch.argsort(code, stable=True)
    qs = qd[order].contiguous()
    view = bvh.view
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)

    def call():
        _lib.call("a3d_udf", ctypes.byref(view), qs.data_ptr(), n, dist_o.data_ptr(), fid_o.data_ptr(),
                  cp_o.data_ptr(), None, None, None, None, _lib.A3D_UDF_ASSUME_SORTED | (flags & ~_lib.A3D_UDF_SORT_QUERIES),
                  ws.data_ptr(), ws.numel(),
                  stream.cuda_stream)

    for _ in range(3):
        call()
    torch.cuda.synchronize()
    ev0.record(stream)
    for _ in range(steps):
        call()
    ev1.record(stream)
    torch.cuda.synchronize()
    return ev0.elapsed_time(ev1) / steps


if __name__ == "__main__":
    main()
