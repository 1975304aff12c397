"""Benchmark of the adaptive SpMV / SpMSpV engine on B200.

Workload (one "step"): the 1,048,576 x 1,048,576 Zipf-row matrix (nnz
16,777,216, row lengths Zipf(1.5) scaled to mean 16, values U(-1,1), seed 2)
multiplied by a sparse x at each density of the sweep 1e-5, 1e-4, 1e-3, 1e-2,
1e-1, 1.0 (positions uniform without replacement, values U(-1,1)); each call
goes through the adaptive engine (selector + chosen kernel).  Synthetic data
of the benchmark's shape: no dataset is involved.

Metric: effective GB/s = compulsory bytes of the cheapest formulation of each
call (min of the CSC SpMSpV traffic 16*x_nnz + 8*bin_len + 4*m and the SpMV
traffic 4(m+1) + 8*nnz + 4n + 4m), summed over the sweep, divided by the
device time of the step (the six calls back to back, CUDA events around them,
the L2 flushed before each step).  `value` has inputs resident in HBM; `e2e`
adds, per call, the host->device copy of x (pinned) and the device->host read
of y: its nonzeros (keys, values and their count, compacted straight into
pinned host memory) for a sparse x, the dense y for the dense x; one stream
synchronisation per step.

--impl reference times the reference's CPU path on all host threads on the
same sweep (the reference's own serialspmv over row slices for the dense x,
the oracle's OpenMP restatement of SpmSpvCSCHost for a sparse x), on inputs
built by the oracle, and the reference's own GPU kernels rebuilt for sm_100a.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(ROOT, "spmspv-adaptive_b200")
for _p in (ROOT, PKG):
    if _p not in sys.path:
        sys.path.insert(0, _p)

import numpy as np  # noqa: E402

METRIC = "SpMSpV/SpMV effective HBM GB/s vs x density; batched BFS GTEPS vs plain"
WORKLOAD = ("zipf-1M density sweep: 1,048,576^2 CSR+CSC, nnz 16,777,216, Zipf(1.5) rows "
            "(mean 16, cap 10,000), x density 1e-5..1.0, adaptive kernel per call")
DENSITIES = (1e-5, 1e-4, 1e-3, 1e-2, 1e-1, 1.0)
SPMV_BACKENDS = {0: "hola", 1: "csr5", 2: "tiled", 3: "round"}


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def eff_bytes(m, n, nnz, x_nnz, bin_len):
    csc = 16 * x_nnz + 8 * bin_len + 4 * m
    spmv = 4 * (m + 1) + 8 * nnz + 4 * n + 4 * m
    return min(csc, spmv)


def spmv_bytes(m, n, nnz):
    return 4 * (m + 1) + 8 * nnz + 4 * n + 4 * m


def ref_spmv_bytes(m, nnz):
    """The reference's own SpMV byte count, SpmvGetBytes (detail/util.h:145):
    row pointers and column indices, then values, x read once per nonzero,
    and y."""
    return (m + 1 + nnz) * 4 + (2 * nnz + m) * 4


def ref_gm1_bytes(x_nnz, bin_len):
    """The reference's traffic model of the CSC SpMSpV, GM1 (csc-spmspv/spmspv.h:2727-2733):
    12 bytes per x entry and 12 per product."""
    return 12 * x_nnz + 12 * bin_len


class Clocks:
    """nvidia-smi sampling during the timed region."""

    def __init__(self, index):
        self.index = index
        self.proc = None
        import tempfile
        self.path = os.path.join(tempfile.gettempdir(), f"spmx_clocks_{os.getpid()}.csv")

    def __enter__(self):
        try:
            os.makedirs(os.path.dirname(self.path), exist_ok=True)
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index),
                 "--query-gpu=clocks.sm,clocks.max.sm,clocks_event_reasons.active,"
                 "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
                 "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=self.f, stderr=subprocess.DEVNULL)
            time.sleep(0.3)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc:
            time.sleep(0.25)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
            self.f.close()

    def summary(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"]}
        rows = []
        with open(self.path) as f:
            for ln in f:
                parts = [p.strip() for p in ln.split(",")]
                if len(parts) >= 7:
                    rows.append(parts)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        sm = [float(r[0]) for r in rows if r[0].replace(".", "").isdigit()]
        mx = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[3 + i] == "Active"})
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": reasons,
                "samples": len(rows)}


def dist_init(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        import torch
        import torch.distributed as dist
        backend = "gloo" if args.impl == "reference" else "nccl"
        if backend == "nccl":
            torch.cuda.set_device(local)
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=120))
    return world, rank, local


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def allmax(v, world):
    if world == 1:
        return v
    import torch
    import torch.distributed as dist
    t = torch.tensor([v], dtype=torch.float64,
                     device="cuda" if dist.get_backend() == "nccl" else "cpu")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def make_inputs():
    """The benchmark's inputs from the product's generators (libspmx.so)."""
    from spmx import gen
    A = gen.zipf_1m(seed=2)
    xs = []
    for d in DENSITIES:
        k = gen.density_nnz(A.n, d)
        key, val = gen.sparse_vector(A.n, k, dist="uniform", seed=1000 + k)
        xs.append((d, key, val))
    return A, xs


def make_inputs_oracle():
    """The same inputs from the oracle's restatement of the generators (bit
    for bit the same, checked by tests/test_gen.py): the CPU reference arm
    loads nothing from the product library."""
    import oracle.oracle as orc
    A = orc.gen_zipf_1m(seed=2)
    xs = []
    for d in DENSITIES:
        k = orc.density_nnz(A.n, d)
        key, val = orc.gen_sparse_vector(A.n, k, "uniform", 1000 + k)
        xs.append((d, key, val))
    return A, xs


def cpu_model():
    """The host CPU's model name (lscpu's "Model name", from /proc/cpuinfo)."""
    try:
        with open("/proc/cpuinfo") as f:
            for ln in f:
                if ln.startswith("model name"):
                    return ln.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def ref_host_libs():
    """The reference's own host routines compiled from its sources
    (oracle/_ref): (libref_host.so with serialspmv, libref_csc.so with
    SpmSpvCSCHost), or None where they were not built."""
    import ctypes
    so1 = os.path.join(ROOT, "oracle", "_ref", "libref_host.so")
    so2 = os.path.join(ROOT, "oracle", "_ref", "libref_csc.so")
    if not (os.path.exists(so1) and os.path.exists(so2)):
        return None
    h, c = ctypes.CDLL(so1), ctypes.CDLL(so2)
    P = ctypes.c_void_p
    h.ref_serialspmv.argtypes = [ctypes.c_int] * 3 + [P] * 5 + [ctypes.c_float]
    h.ref_serialspmv.restype = None
    h.ref_serialspmv_slices.argtypes = [ctypes.c_int, P] + [ctypes.c_int] * 3 + [P] * 5 + [ctypes.c_float]
    h.ref_serialspmv_slices.restype = None
    c.ref_spmspv_csc_host.argtypes = [ctypes.c_int] * 3 + [P] * 3 + [ctypes.c_int] + [P] * 5
    c.ref_spmspv_csc_host.restype = None
    return h, c


def row_slices(rowptr, parts):
    """Row ranges with about nnz/parts nonzeros each."""
    nnz = int(rowptr[-1])
    cuts = np.searchsorted(rowptr, np.linspace(0, nnz, parts + 1)[1:-1]).tolist()
    b = [0] + cuts + [len(rowptr) - 1]
    return [(b[i], b[i + 1]) for i in range(parts) if b[i + 1] > b[i]]


def ref_gpu_sweep(A, xs, colptr, row, cval, binl, reps=7):
    """The reference's own GPU kernels (oracle/_ref, rebuilt for sm_100a from
    its sources) on the same sweep: per density the fastest of the kernels
    that run here (CSC naive atomic SpMSpV for every density; Hola and naive
    CSR SpMV for the dense x), each result checked against the FP64 oracle.
    Left out: the merge-path and sort CSC SpMSpV, whose chained scan spins
    without a bound on the previous block's sum, and CSR5, whose descriptor
    kernel writes one word past its descriptor array on this matrix (a row
    starting at offset nnz, with nnz a multiple of 32 * sigma); the
    comparator library does not contain that path."""
    import ctypes
    import oracle.oracle as orc
    so = os.path.join(ROOT, "oracle", "_ref", "libref_host.so")
    if not os.path.exists(so):
        return {"unavailable": "oracle/_ref/libref_host.so not built"}
    lib = ctypes.CDLL(so)
    if lib.ref_gpu_count() < 1:
        return {"unavailable": "no CUDA device visible to the reference's GPU kernels"}
    P = ctypes.c_void_p
    lib.ref_gpu_time.argtypes = [ctypes.c_int] * 4 + [P] * 7 + [ctypes.c_int, P, P, ctypes.c_int, P, P]
    lib.ref_gpu_time.restype = ctypes.c_int
    m, n, nnz = A.m, A.n, A.nnz
    names = {0: "hola-spmv", 2: "naive-spmv", 3: "csc-naive-atomic"}
    per = []
    tot_ms, tot_bytes = 0.0, 0
    for (d, key, val), b in zip(xs, binl):
        xd = orc.sparse2dense_bits(n, key, val)[0].astype(np.float32)
        y64, mag = orc.spmv_f64(A.rowptr, A.col, A.val, xd)
        kinds = (3, 0, 2) if d >= 1.0 else (3,)
        times = {}
        for w in kinds:
            ms = np.zeros(reps, np.float32)
            y = np.zeros(m, np.float32)
            rc = lib.ref_gpu_time(w, m, n, nnz, A.rowptr.ctypes.data, A.col.ctypes.data, A.val.ctypes.data,
                                  colptr.ctypes.data, row.ctypes.data, cval.ctypes.data, xd.ctypes.data,
                                  len(key), key.ctypes.data, val.ctypes.data, reps, ms.ctypes.data,
                                  y.ctypes.data)
            ok = rc == 0 and bool(orc.within_tol(y, y64, mag, 1e-5)[0])
            times[names[w]] = {"ms": float(np.median(ms)), "within_1e-5": ok}
        good = [(v["ms"], k) for k, v in times.items() if v["within_1e-5"]]
        if not good:
            per.append({"density": d, "best": None, "kernels": times})
            continue
        best = min(good)
        per.append({"density": d, "best": best[1], "ms": best[0], "kernels": times})
        tot_ms += best[0]
        tot_bytes += eff_bytes(m, n, nnz, len(key), b)
    if any(p["best"] is None for p in per):
        return {"unavailable": "a density had no result within 1e-5", "sweep": per}
    return {"value": tot_bytes / (tot_ms * 1e-3) / 1e9, "unit": "GB/s", "ms_per_step": tot_ms,
            "what": "the reference's kernels rebuilt for sm_100a, fastest correct one per density "
                    "(an exhaustive pick, no selector cost), L2 flushed before each call",
            "sweep": per}


# ---------------------------------------------------------------------------
# reference arm: the reference's CPU routines on all host threads
# ---------------------------------------------------------------------------
def run_reference(args, world, rank):
    """The reference arm: the reference's CPU path on all host threads, on
    inputs built by the oracle (nothing of the product is loaded).  The dense
    leg is the reference's own serialspmv (oracle/_ref, compiled from its
    sources), run over nnz-balanced row slices on every host thread; the
    sparse legs are the oracle's OpenMP restatement of SpmSpvCSCHost (x
    entries across threads, atomic adds), because the reference's routine is
    one serial loop into one dense y and cannot be split without changing it.
    With --ref-gpu (the default) the line also carries the reference's own GPU
    kernels rebuilt for sm_100a on the same sweep."""
    if rank != 0:
        return 0
    import oracle.oracle as orc
    A, xs = make_inputs_oracle()
    colptr, row, cval = A.to_csc()
    threads = orc.raw.cpu_threads()
    m, n, nnz = A.m, A.n, A.nnz
    y = np.zeros(m, np.float32)
    P = lambda a: a.ctypes.data  # noqa: E731
    binl = [int(orc.vec_features(colptr, key)[0]) for _, key, _ in xs]
    tot_bytes = sum(eff_bytes(m, n, nnz, len(k), b) for (_, k, _), b in zip(xs, binl))
    dense = [orc.sparse2dense_bits(n, k, v)[0] for _, k, v in xs]
    libs = ref_host_libs()
    slices = row_slices(A.rowptr, 8 * threads)  # several per thread: dynamic scheduling balances
    bounds = np.array([a for a, _ in slices] + [slices[-1][1]], np.int32)

    def dense_leg(xd):
        if libs is None:
            orc.raw.cpu_spmv_omp(m, P(A.rowptr), P(A.col), P(A.val), P(xd), P(y), 1.0)
            return
        # the reference's serialspmv on each slice, an OpenMP loop over the slices
        libs[0].ref_serialspmv_slices(len(slices), P(bounds), m, n, nnz, P(A.rowptr), P(A.col), P(A.val),
                                      P(xd), P(y), 1.0)

    def step():
        t = 0.0
        for (d, key, val), xd in zip(xs, dense):
            t0 = time.perf_counter()
            if d >= 1.0:
                dense_leg(xd)
            else:
                orc.raw.cpu_spmspv_csc_omp(m, P(colptr), P(row), P(cval), len(key), P(key),
                                           P(val), P(y))
            t += time.perf_counter() - t0
        return t

    for _ in range(args.warmup):
        step()
    ts = [step() for _ in range(args.steps)]
    sec = sum(ts) / len(ts)
    gbs = tot_bytes / sec / 1e9
    dense_what = ("the reference's own serialspmv (oracle/_ref) over %d nnz-balanced row slices, an "
                  "OpenMP loop on %d host threads" % (len(slices), threads)) if libs else \
        "the oracle's serialspmv, OpenMP"
    line = {"metric": METRIC, "value": gbs, "unit": "GB/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": sec * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic", "impl": "reference",
            "config": {"workload": WORKLOAD, "parallelism": "replicas" if args.gpus > 1 else "single"},
            "cpu_baseline": {"value": gbs, "unit": "GB/s", "cores": threads, "cpu": cpu_model(),
                             "kind": "port",
                             "sample": "the full 6-density sweep per step; dense x: " + dense_what +
                                       "; sparse x: SpmSpvCSCHost restated (oracle), OpenMP over all "
                                       "host threads"},
            "e2e": {"value": gbs, "unit": "GB/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    if not args.no_ref_gpu:
        line["ref_gpu_sm100a"] = ref_gpu_sweep(A, xs, colptr, row, cval, binl)
    print(json.dumps(line), flush=True)
    return 0


# ---------------------------------------------------------------------------
# our arm
# ---------------------------------------------------------------------------
def run_ours(args, world, rank, local):
    import torch
    import spmx
    from spmx import abi
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    # one side stream for everything (graph capture needs a stream other than
    # the legacy default stream)
    stream = torch.cuda.Stream(dev)
    torch.cuda.set_stream(stream)
    A, xs = make_inputs()
    m, n, nnz = A.m, A.n, A.nnz

    def d(a):
        return torch.from_numpy(np.ascontiguousarray(a)).to(dev)

    rp, cl, vl = d(A.rowptr), d(A.col), d(A.val)
    h = spmx.SpmspvHandle(m, n, nnz, stream=stream)
    h.InputCSR(nnz, rp, cl, vl)
    h.ToCSC()
    h.holaPreprocess()
    h.allocPreBuffer()
    spmv_type = h.autotune(args.tune_cache)  # per-matrix launch parameters and SpMV back-end (untimed)
    xdense = torch.zeros(n, device=dev)
    bits = torch.zeros((n + 31) // 32, dtype=torch.int32, device=dev)
    h.set_x(xdense)
    h.set_bitvector(bits, (n + 31) // 32)
    y = torch.empty(m, device=dev)
    dx = [(dd, d(k), d(v), len(k)) for dd, k, v in xs]
    binl = []
    for dd, kd, vd, k in dx:
        h.set_sparse_x(kd, vd, k)
        binl.append(h.computeBinlenVer2())
    ebytes = [eff_bytes(m, n, nnz, k, b) for (_, _, _, k), b in zip(dx, binl)]
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=dev)  # 256 MiB > L2

    # --- one step = the whole sweep: the six adaptive calls through the public
    # API, back to back on one stream, each into its own y (the selector picks
    # every call's kernel on the host, from features it knows without a device
    # round trip); one pair of CUDA events around the step, the L2 flushed
    # before it.  The timed region holds device work only: after the flush the
    # GPU also spins for about 100 us (outside the events), so the host has
    # enqueued all six calls before the start event.  Enqueueing a call through
    # the Python binding costs about 10 us of host time, more than the small
    # densities take on the device, so without that head start a slow host
    # leaves the GPU waiting inside the step; `ms_per_step_host_paced` is the
    # same step with the flush alone. ---
    ys = [torch.empty(m, device=dev) for _ in dx]
    chosen = [None] * len(dx)
    s_ev, e_ev = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    head_start_cycles = 200_000  # ~100 us at 1,965 MHz

    def step(head_start=True):
        flush.fill_(1.0)
        if head_start:
            torch.cuda._sleep(head_start_cycles)
        s_ev.record(stream)
        for i, (dd, kd, vd, k) in enumerate(dx):
            h.set_sparse_x(kd, vd, k)
            chosen[i] = h.run_adaptive(1.0, ys[i])
        e_ev.record(stream)
        stream.synchronize()
        return s_ev.elapsed_time(e_ev)

    for _ in range(max(args.warmup, 3)):
        step()
    h.check_device_error()
    barrier(world)
    torch.cuda.synchronize(dev)
    step_t = []
    l0 = abi.lib.spmx_launch_count()
    with Clocks(local) as clk:
        for _ in range(args.steps):
            step_t.append(step())
    launches = abi.lib.spmx_launch_count() - l0
    launches_per_step = launches // max(args.steps, 1)
    torch.cuda.synchronize(dev)
    barrier(world)
    h.check_device_error()
    step_ms = float(np.mean(step_t))
    step_ms_max = allmax(step_ms, world)
    paced_t = [step(head_start=False) for _ in range(args.steps)]
    paced_ms = allmax(float(np.mean(paced_t)), world)
    total_bytes = float(sum(ebytes))
    value = world * total_bytes / (step_ms_max * 1e-3) / 1e9
    # the timed replays' results, kept for the check against the oracle below
    ys_h = [t.cpu().numpy().astype(np.float64) for t in ys]

    # --- each call alone, the L2 flushed before it (CUDA events around the
    # call; an empty kernel timed this way after the flush takes about 6 us) ---
    ev1 = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in dx]
    per_call = np.zeros(len(dx))
    for it in range(3 + args.steps):
        for i, (dd, kd, vd, k) in enumerate(dx):
            flush.fill_(float(i))
            h.set_sparse_x(kd, vd, k)
            ev1[i][0].record(stream)
            h.run_adaptive(1.0, y)
            ev1[i][1].record(stream)
        stream.synchronize()
        if it >= 3:
            per_call += np.array([a.elapsed_time(b) for a, b in ev1])
    per_call /= args.steps
    # --- each call's share of the chained step: the step cut after call k
    # (the same flush, events and calls as a step), minus the step cut after
    # call k - 1; the first share includes the cost of the step's first launch
    # after the flush ---
    prefix = np.zeros(len(dx))
    for it in range(3 + args.steps):
        for kk in range(1, len(dx) + 1):
            flush.fill_(1.0)
            torch.cuda._sleep(head_start_cycles)
            s_ev.record(stream)
            for i in range(kk):
                h.set_sparse_x(dx[i][1], dx[i][2], dx[i][3])
                h.run_adaptive(1.0, ys[i])
            e_ev.record(stream)
            stream.synchronize()
            if it >= 3:
                prefix[kk - 1] += s_ev.elapsed_time(e_ev)
    prefix /= args.steps
    in_step = np.diff(np.concatenate([[0.0], prefix]))
    # the same timing around a kernel that writes one float: what an event
    # pair around any single launch costs after the flush
    tiny = torch.zeros(1, device=dev)
    floor_t = []
    for it in range(3 + args.steps):
        flush.fill_(float(it))
        ev1[0][0].record(stream)
        tiny.fill_(float(it))
        ev1[0][1].record(stream)
        stream.synchronize()
        if it >= 3:
            floor_t.append(ev1[0][0].elapsed_time(ev1[0][1]))
    floor_ms = statistics.median(floor_t)

    # --- roofline: the load-balanced SpMV on the dense x (the dominant call of
    # the sweep), through the dispatcher, i.e. the back-end the autotuner chose
    h.set_sparse_x(dx[-1][1], dx[-1][2], dx[-1][3])
    h.sparse2dense()
    rs, re_ = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    kt = []
    for it in range(args.warmup + args.steps):
        flush.fill_(1.0)
        rs.record(stream)
        h.spmv(1.0, y)
        re_.record(stream)
        stream.synchronize()
        if it >= args.warmup:
            kt.append(rs.elapsed_time(re_))
    k_ms = statistics.mean(kt)
    sb = spmv_bytes(m, n, nnz)
    peak, peak_kind = peaks()
    achieved = sb / (k_ms * 1e-3) / 1e9
    kname = SPMV_BACKENDS.get(spmv_type, str(spmv_type))
    traffic = None
    tp = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(tp):
        with open(tp) as f:
            traffic = json.load(f).get(f"{kname}_spmv_zipf1m")
    # what the chosen back-end's own format costs: a rebuild, timed on the
    # host around a synchronised call, and the bytes of its stream
    backend_cost = None
    if kname == "round":
        info0 = h.round_info()
        torch.cuda.synchronize(dev)
        t0 = time.perf_counter()
        h.roundPreprocess(0, info0["parts"])
        torch.cuda.synchronize(dev)
        prep_ms = (time.perf_counter() - t0) * 1e3
        info1 = h.round_info()
        fmt_bytes = info1["rounds"] * 4096 * 8 + info1["rounds"] * 32 * 4 + 4 * (m + 1)
        backend_cost = {"preprocess_ms": prep_ms, "format_bytes": fmt_bytes, "geometry": info1,
                        "csr_bytes": 4 * (m + 1) + 8 * nnz,
                        "spmv_calls_to_amortise": prep_ms / k_ms}

    # --- correctness of the sweep (rank 0): each density's y against the FP64
    # oracle with the parity tests' magnitude-scaled bound, plus the raw
    # relative and normwise errors ---
    correctness = []
    ref64 = []
    import oracle.oracle as orc
    if rank == 0:
        colptr_h, row_h, cval_h = A.to_csc()
        for (dd, kd, vd, k), (_, key, val), yh in zip(dx, xs, ys_h):
            y64, mag, _ = orc.spmspv_csc_f64(m, colptr_h, row_h, cval_h, key, val)
            ref64.append((y64, mag))
            nz = y64 != 0
            rel = float(np.max(np.abs(yh[nz] - y64[nz]) / np.abs(y64[nz]))) if nz.any() else 0.0
            top = float(np.max(np.abs(y64))) if len(y64) else 0.0
            correctness.append({"density": dd, "within_1e-5": bool(orc.within_tol(yh, y64, mag, 1e-5)[0]),
                                "max_scaled_err": orc.max_scaled_err(yh, y64, mag), "max_rel_err": rel,
                                "normwise_err": float(np.max(np.abs(yh - y64))) / top if top else 0.0})
        h.check_device_error()

    # --- e2e through the public API with host buffers, one step = the sweep.
    # The inputs sit in pinned host memory in two packed buffers, each x as
    # its keys followed by its values: the five smaller x together, and the
    # largest x (the dense-x call) alone.  A copy of any size costs ~15-20 us
    # of fixed time on this link, so two copies replace twelve.  The small
    # buffer goes first (1.3 MB), so the five small calls run while the 8 MB
    # one is still uploading.  Each call waits on an event for its own buffer
    # only.  Results come back without a host round trip, on a read-back
    # stream that waits for each call's event, so the calls queued behind a
    # read-back do not wait for it (every call has its own y): for a sparse x,
    # spmx_dense2sparse_to_host compacts y's nonzeros and their count straight
    # into pinned host memory (the handle's stream is switched to the
    # read-back stream for that call: the compaction's only scratch is its
    # per-range counts, which no SpMV/SpMSpV call uses, and the compactions run
    # one after another on that stream); the dense y is copied.  One stream
    # synchronisation per step; the L2 is flushed between steps.
    big = [int(np.argmax([len(k) for _, k, _ in xs]))]
    rest = [i for i in range(len(xs)) if i not in big]
    groups = [g for g in (rest, big) if g]

    def packed(group):
        tot = sum(2 * len(xs[i][1]) for i in group)
        hb = torch.empty(max(tot, 1), dtype=torch.int32).pin_memory()
        db = torch.empty(max(tot, 1), dtype=torch.int32, device=dev)
        views, o = {}, 0
        for i in group:
            k = len(xs[i][1])
            hb[o:o + k] = torch.from_numpy(np.ascontiguousarray(xs[i][1]))
            hb[o + k:o + 2 * k] = torch.from_numpy(np.ascontiguousarray(xs[i][2])).view(torch.int32)
            views[i] = (db[o:o + k], db[o + k:o + 2 * k].view(torch.float32))
            o += 2 * k
        return hb, db, views

    packs = [packed(g) for g in groups]
    xview = {i: v for _, _, vw in packs for i, v in vw.items()}
    sparse_out = [dd < 1.0 for dd, _, _ in xs]
    yhost = torch.empty(m, dtype=torch.float32).pin_memory()
    ykey_h = [torch.empty(m if sp else 1, dtype=torch.int32).pin_memory() for sp in sparse_out]
    yval_h = [torch.empty(m if sp else 1, dtype=torch.float32).pin_memory() for sp in sparse_out]
    ycnt_h = torch.zeros(len(xs), dtype=torch.int32).pin_memory()
    h2d = sum(8 * len(k) for _, k, _ in xs)
    d2h_calls = []
    e2e_ok = []
    copy_stream, d2h_stream = torch.cuda.Stream(dev), torch.cuda.Stream(dev)
    ev_in = [torch.cuda.Event() for _ in groups]
    ev_done = [torch.cuda.Event() for _ in xs]
    ev_back = torch.cuda.Event()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)

    def e2e_step(check=False):
        flush.fill_(2.0)
        e0.record(stream)
        copy_stream.wait_event(e0)
        d2h_stream.wait_event(e0)
        with torch.cuda.stream(copy_stream):
            for (hb, db, _), ev in zip(packs, ev_in):
                db.copy_(hb, non_blocking=True)
                ev.record(copy_stream)
        for g, ev in zip(groups, ev_in):
            stream.wait_event(ev)
            for i in g:
                kd, vd = xview[i]
                h.set_sparse_x(kd, vd, len(xs[i][1]))
                h.run_adaptive(1.0, ys[i])
                ev_done[i].record(stream)
                d2h_stream.wait_event(ev_done[i])
                if sparse_out[i]:
                    h.set_stream(d2h_stream)
                    h.dense2sparse_to_host(m, ys[i], ykey_h[i], yval_h[i], ycnt_h[i:i + 1])
                    h.set_stream(stream)
                else:
                    with torch.cuda.stream(d2h_stream):
                        yhost.copy_(ys[i], non_blocking=True)
        ev_back.record(d2h_stream)
        stream.wait_event(ev_back)
        e1.record(stream)
        stream.synchronize()
        d2h_calls.clear()
        for i in range(len(xs)):
            ynz = int(ycnt_h[i]) if sparse_out[i] else m
            d2h_calls.append(4 + 8 * ynz if sparse_out[i] else 4 * m)
            if check and ref64:
                got = np.zeros(m, np.float64)
                if sparse_out[i]:
                    got[ykey_h[i][:ynz].numpy()] = yval_h[i][:ynz].numpy()
                else:
                    got[:] = yhost.numpy()
                e2e_ok.append(bool(orc.within_tol(got, ref64[i][0], ref64[i][1], 1e-5)[0]))
        return e0.elapsed_time(e1)

    for _ in range(max(args.warmup, 3)):
        e2e_step()
    barrier(world)
    e2e_ms = statistics.mean([e2e_step() for _ in range(args.steps)])
    e2e_ms = allmax(e2e_ms, world)
    d2h = sum(d2h_calls)
    e2e_val = world * total_bytes / (e2e_ms * 1e-3) / 1e9
    e2e_step(check=True)  # untimed: the host-side results against the FP64 oracle

    # The PCIe share of e2e: the same bytes moved by copies alone, the two
    # uploads on the copy stream and the read-backs (one per array the step
    # returns) on the read-back stream, so that both directions run at once.
    ynz_last = [int(ycnt_h[i]) if sparse_out[i] else m for i in range(len(xs))]

    def copies_step():
        flush.fill_(2.0)
        e0.record(stream)
        copy_stream.wait_event(e0)
        d2h_stream.wait_event(e0)
        with torch.cuda.stream(copy_stream):
            for hb, db, _ in packs:
                db.copy_(hb, non_blocking=True)
            ev_in[0].record(copy_stream)
        with torch.cuda.stream(d2h_stream):
            for i in range(len(xs)):
                nz = ynz_last[i]
                if sparse_out[i]:
                    ycnt_h[i:i + 1].copy_(ycnt_d[i:i + 1], non_blocking=True)
                    ykey_h[i][:nz].copy_(ys[i][:nz].view(torch.int32), non_blocking=True)
                    yval_h[i][:nz].copy_(ys[i][:nz], non_blocking=True)
                else:
                    yhost.copy_(ys[i], non_blocking=True)
            ev_back.record(d2h_stream)
        stream.wait_event(ev_in[0])
        stream.wait_event(ev_back)
        e1.record(stream)
        stream.synchronize()
        return e0.elapsed_time(e1)

    ycnt_d = torch.zeros(len(xs), dtype=torch.int32, device=dev)
    for _ in range(3):
        copies_step()
    copies_ms = allmax(statistics.mean([copies_step() for _ in range(args.steps)]), world)

    # --- the selector against exhaustive timing of all eight kernels (rank 0,
    # after the last collective) ---
    exhaustive = []
    if rank == 0:
        from spmx import KERNEL_NAMES
        for i, (dd, kd, vd, k) in enumerate(dx):
            h.set_sparse_x(kd, vd, k)
            times = []
            for kid in range(len(KERNEL_NAMES)):
                ts = []
                for it in range(7):
                    flush.fill_(float(it))
                    rs.record(stream)
                    h.run_kernel(kid, 1.0, y)
                    re_.record(stream)
                    stream.synchronize()
                    if it >= 2:
                        ts.append(rs.elapsed_time(re_))
                times.append(statistics.median(ts))
            best = int(np.argmin(times))
            exhaustive.append({"density": dd, "chosen": KERNEL_NAMES[chosen[i]], "best": KERNEL_NAMES[best],
                               "regret": times[chosen[i]] / times[best],
                               "ms": {KERNEL_NAMES[j]: round(t, 4) for j, t in enumerate(times)}})
        h.check_device_error()

    # --- BFS on R-MAT scale 14 (plain), bit-exact check against the oracle ---
    bfs = run_bfs_plain(torch, dev, stream, args) if rank == 0 and not args.no_bfs else None
    bfs64 = run_bfs_batched(torch, dev, stream, args) if rank == 0 and not args.no_bfs else None
    batched = run_batched_spmspv(torch, dev, stream, args) if rank == 0 and not args.no_batched else None
    adjoint = run_adjoint(torch, dev, stream, args) if rank == 0 and not args.no_batched else None
    ingest = run_ingest(torch, dev, stream, args) if rank == 0 and not args.no_ingest else None
    hybrid = run_hybrid(torch, dev, stream, args) if rank == 0 and not args.no_batched else None
    powerlaw = run_powerlaw(torch, dev, stream, args) if rank == 0 and not args.no_batched else None

    line = None
    if rank == 0:
        cpu = cpu_baseline(A, xs, binl) if not args.no_cpu and world == 1 else None
        sweep = [{"density": dd, "x_nnz": k, "bin_len": b, "kernel": abi.KERNEL_NAMES[c],
                  "ms_alone_flushed": float(t1), "eff_gbs_alone_flushed": eb / (t1 * 1e-3) / 1e9,
                  "ms_in_step": float(t2), "bytes_compulsory": int(eb),
                  "bytes_reference_gm1": int(ref_gm1_bytes(k, b))}
                 for (dd, _, _, k), b, c, t1, eb, t2 in zip(dx, binl, chosen, per_call, ebytes, in_step)]
        line = {
            "metric": METRIC, "value": value, "unit": "GB/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": step_ms_max,
            "ms_per_step_host_paced": paced_ms,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic",
            "config": {"workload": WORKLOAD,
                       "step": "the six adaptive calls of the sweep, back to back through the public API",
                       "l2": "flushed (256 MiB write) before every timed step",
                       "row_lengths": {"mean": float(np.mean(np.diff(A.rowptr))),
                                       "max": int(np.max(np.diff(A.rowptr))),
                                       "std": float(np.std(np.diff(A.rowptr)))},
                       "spmv_backend": kname,
                       "parallelism": f"replicas x{world}" if world > 1 else "single"},
            "spmv_backend_cost": backend_cost,
            "roofline": {"bound": "hbm", "kernel": f"{kname} SpMV (autotuned back-end), dense x",
                         "achieved": achieved, "peak": peak, "peak_kind": peak_kind,
                         "unit": "GB/s", "frac": achieved / peak, "traffic": traffic,
                         "bytes_per_launch": sb, "ms_per_launch": k_ms,
                         "reference_bytes_per_launch": ref_spmv_bytes(m, nnz),
                         "achieved_reference_bytes_gbs": ref_spmv_bytes(m, nnz) / (k_ms * 1e-3) / 1e9,
                         "ms_per_launch_median": statistics.median(kt), "ms_per_launch_min": min(kt)},
            "e2e": {"value": e2e_val, "unit": "GB/s", "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h, "ms_per_step": e2e_ms,
                    "copies_only_ms": copies_ms, "input_copies": len(packs),
                    "host_results_within_1e-5": bool(e2e_ok) and all(e2e_ok)},
            "gpu_launches": int(launches),
            "gpu_launches_per_step": int(launches_per_step),
            "clocks": clk.summary(),
            "sweep": sweep,
            "one_kernel_floor_ms": floor_ms,
            "correctness": correctness,
            "selector_vs_exhaustive": exhaustive,
            "cpu_baseline": cpu,
            "bfs": bfs,
            "batched_bfs": bfs64,
            "batched_spmspv": batched,
            "adjoint": adjoint,
            "ingest": ingest,
            "hybrid_candidate": hybrid,
            "powerlaw_spmv": powerlaw,
        }
        print(json.dumps(line), flush=True)
    h.Destroy()
    return 0


def run_bfs_plain(torch, dev, stream, args):
    """R-MAT scale 14 (edge factor 16, seed 1) from vertex 0: one traversal
    per timed call (one cooperative launch, no read-back, as in the batched
    comparison), L2 flushed before each."""
    import spmx
    from spmx import gen
    import oracle.oracle as orc
    g = gen.rmat(14, 16, seed=1)
    rp = torch.from_numpy(g.rowptr).to(dev)
    cl = torch.from_numpy(g.col).to(dev)
    h = spmx.SpmspvHandle(g.m, g.n, g.nnz, stream=stream)
    h.InputCSR(g.nnz, rp, cl, None)
    lv = torch.empty(g.n, dtype=torch.int32, device=dev)
    s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=dev)  # the graph fits in L2
    for _ in range(3):
        h.bfs(0, lv)
    ts = []
    for it in range(max(args.steps, 5)):
        flush.fill_(float(it))
        s.record(stream)
        h.bfs(0, lv, sync=False)  # the traversal; the depth is read once below
        e.record(stream)
        stream.synchronize()
        ts.append(s.elapsed_time(e))
    depth = h.bfs(0, lv)
    ref, _ = orc.bfs_queue(g.n, g.rowptr, g.col, 0)
    got = lv.cpu().numpy()
    reached = ref >= 0
    # Graph500 convention: undirected input edges inside the source's component
    edges = int(np.diff(g.rowptr)[reached].sum()) // 2
    ms = statistics.median(ts)
    h.Destroy()
    return {"graph": "rmat scale 14, edge factor 16, seed 1, source 0",
            "ms": ms, "gteps": edges / (ms * 1e-3) / 1e9, "depth": depth,
            "bit_exact": bool(np.array_equal(got, ref)), "edges": edges,
            "gteps_edges": "undirected input edges inside the source's component (Graph500)"}


def run_bfs_batched(torch, dev, stream, args):
    """R-MAT scale 22 (edge factor 16, seed 3), 64 sources drawn (seed 3) from
    vertices of degree > 0: one batched launch vs 64 plain traversals."""
    import spmx
    from spmx import gen
    g = gen.rmat(22, 16, seed=3)
    rng = np.random.default_rng(3)
    deg = np.diff(g.rowptr)
    srcs = rng.choice(np.nonzero(deg > 0)[0], 64, replace=False).tolist()
    rp = torch.from_numpy(g.rowptr).to(dev)
    cl = torch.from_numpy(g.col).to(dev)
    h = spmx.SpmspvHandle(g.m, g.n, g.nnz, stream=stream)
    h.InputCSR(g.nnz, rp, cl, None)
    n = g.n
    lv_b = torch.empty(64 * n, dtype=torch.int32, device=dev)
    lv_p = torch.empty(64 * n, dtype=torch.int32, device=dev)
    s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    reps = 3
    h.bfs_batched(srcs, lv_b, layout=1)
    tb = []
    for _ in range(reps):
        s.record(stream)
        h.bfs_batched(srcs, lv_b, layout=1, sync=False)
        e.record(stream)
        stream.synchronize()
        tb.append(s.elapsed_time(e))
    for i, src in enumerate(srcs[:2]):
        h.bfs(src, lv_p[i * n:(i + 1) * n])
    tp = []
    for _ in range(reps):
        s.record(stream)
        for i, src in enumerate(srcs):
            h.bfs(src, lv_p[i * n:(i + 1) * n], sync=False)
        e.record(stream)
        stream.synchronize()
        tp.append(s.elapsed_time(e))
    h.check_device_error()
    exact = bool(torch.equal(lv_b, lv_p))
    # full-size parity: sampled sources of the batch against the oracle's
    # queue BFS on the host (bit for bit)
    import oracle.oracle as orc
    sampled = (0, 21, 42, 63)
    lvh = lv_b.view(64, n)
    oracle_ok = all(np.array_equal(lvh[i].cpu().numpy(), orc.bfs_queue(n, g.rowptr, g.col, srcs[i])[0])
                    for i in sampled)
    degd = torch.from_numpy(deg.astype(np.int64)).to(dev)
    reached = (lv_p.view(64, n) >= 0).to(torch.int64)
    edges = int((reached * degd).sum().item()) // 2
    mb, mp = statistics.median(tb), statistics.median(tp)
    h.Destroy()
    return {"graph": "rmat scale 22, edge factor 16, seed 3, 64 sources (seed 3)",
            "batched_ms": mb, "plain64_ms": mp, "edges": edges,
            "gteps_edges": "undirected input edges inside each source's component, summed over the 64 (Graph500)",
            "batched_gteps": edges / (mb * 1e-3) / 1e9, "plain64_gteps": edges / (mp * 1e-3) / 1e9,
            "speedup": mp / mb, "bit_exact_vs_plain": exact,
            "bit_exact_vs_oracle": {"sources": [int(srcs[i]) for i in sampled], "ok": bool(oracle_ok)}}


def run_batched_spmspv(torch, dev, stream, args):
    """Batched forward + adjoint SpMSpV: Chung-Lu power-law matrix (n 4,194,304,
    degree exponent 2.1, average degree 32, values N(0,1), seed 5) and 256
    sparse x with nnz log-uniform in [10, 100,000] (N(0,1) values, distinct
    uniform positions).  One CUDA graph holds the forward Y = A X (m x 256)
    and the backward (dxval, dvals) for a fixed upstream dY; it is timed
    against 256 sequential single-vector calls (adaptive SpMSpV forward into a
    dense y, one-vector backward without dvals: less work than the batch)."""
    import spmx
    from spmx import gen
    import oracle.oracle as orc
    nvec = 256
    A = gen.chung_lu(1 << args.batched_log2n, 2.1, 32.0, seed=5)
    m, n = A.m, A.n
    rng = np.random.default_rng(5)
    sizes = np.exp(rng.uniform(np.log(10), np.log(100000), nvec)).astype(np.int64)
    keys, vals = [], []
    for v, k in enumerate(sizes):
        kk, vv = gen.sparse_vector(n, int(k), dist="normal", seed=50000 + v)
        keys.append(kk)
        vals.append(vv)
    xptr = np.zeros(nvec + 1, np.int32)
    xptr[1:] = np.cumsum(sizes)
    xkey = np.concatenate(keys).astype(np.int32)
    xval = np.concatenate(vals).astype(np.float32)
    colptr_h = None
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)  # noqa: E731
    h = spmx.SpmspvHandle(m, n, A.nnz, stream=stream)
    h.InputCSR(A.nnz, t(A.rowptr), t(A.col), t(A.val))
    h.ToCSC()
    xp, xk, xv = t(xptr), t(xkey), t(xval)
    gen_t = torch.Generator(device=dev)
    gen_t.manual_seed(5)
    dY = torch.randn((m, nvec), device=dev, generator=gen_t)
    Y = torch.empty((m, nvec), device=dev)
    tot = int(xptr[-1])
    dxval = torch.empty(len(xkey), device=dev)
    dvals = torch.empty(A.nnz, device=dev)
    s = torch.cuda.Stream(device=dev)
    h.set_stream(s)
    # the backward reuses the forward's inversion of the batch and accumulates
    # dxval in the dvals pass (atomic adds: dxval not bitwise reproducible)
    from spmx import abi
    h.set_batch_options(abi.BATCH_REUSE_INVERSION | abi.BATCH_FUSED_DXVAL)
    with torch.cuda.stream(s):
        h.spmspv_batched(xp, xk, xv, 1.0, Y, x_total=tot)
        h.spmspv_batched_backward(xp, xk, xv, 1.0, dY, dxval, dvals, x_total=tot)
    s.synchronize()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g, stream=s):
        h.spmspv_batched(xp, xk, xv, 1.0, Y, x_total=tot)
        h.spmspv_batched_backward(xp, xk, xv, 1.0, dY, dxval, dvals, x_total=tot)
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    reps = max(args.steps, 5)
    with torch.cuda.stream(s):
        for _ in range(3):
            g.replay()
        tb = []
        for _ in range(reps):
            ev0.record(s)
            g.replay()
            ev1.record(s)
            s.synchronize()
            tb.append(ev0.elapsed_time(ev1))
    h.check_device_error()
    # parity on sampled vectors (forward) against the FP64 oracle
    colptr_h, row_h, cval_h = A.to_csc()
    Yh = None
    ok = True
    for v in (0, nvec // 2, int(np.argmax(sizes))):
        a, b = xptr[v], xptr[v + 1]
        y64, mag, _ = orc.spmspv_csc_f64(m, colptr_h, row_h, cval_h, xkey[a:b], xval[a:b])
        Yh = Y[:, v].cpu().numpy()
        ok = ok and orc.within_tol(Yh, y64, mag, 1e-5)[0]
    # backward parity at full size: dxval of the sampled vectors against FP64
    # A^T dy over the whole matrix, dvals on 4,096 sampled nonzeros against
    # FP64 sums over the batch's entries in their column
    bwd_ok = True
    for v in (0, nvec // 2, int(np.argmax(sizes))):
        a, b = xptr[v], xptr[v + 1]
        dx64, adx = orc.spmv_t_f64(n, A.rowptr, A.col, A.val, dY[:, v].cpu().numpy())
        kk = xkey[a:b]
        bwd_ok = bwd_ok and orc.within_tol(dxval[a:b].cpu().numpy(), dx64[kk], adx[kk], 1e-5)[0]
    ks = np.sort(rng.choice(A.nnz, 4096, replace=False))
    rows_k = np.searchsorted(A.rowptr, ks, side="right") - 1
    cols_k = A.col[ks]
    order = np.argsort(xkey, kind="stable")
    skey = xkey[order]
    svec = np.repeat(np.arange(nvec), sizes)[order]
    sval = xval[order].astype(np.float64)
    dyr = dY[torch.from_numpy(rows_k).to(dev)].cpu().numpy().astype(np.float64)  # 4,096 x nvec
    lo, hi = np.searchsorted(skey, cols_k, "left"), np.searchsorted(skey, cols_k, "right")
    dv64, dvmag = np.zeros(len(ks)), np.zeros(len(ks))
    for i in range(len(ks)):
        terms = sval[lo[i]:hi[i]] * dyr[i, svec[lo[i]:hi[i]]]
        dv64[i], dvmag[i] = terms.sum(), np.abs(terms).sum()
    got_dv = dvals[torch.from_numpy(ks).to(dev)].cpu().numpy()
    bwd_ok = bool(bwd_ok and orc.within_tol(got_dv, dv64, dvmag, 1e-5)[0])
    bins = int(np.sum(colptr_h[xkey + 1] - colptr_h[xkey]))
    h.set_batch_options(0)
    # 256 sequential single-vector calls: the forward through the adaptive
    # single-vector engine (selector + CSC SpMSpV into a dense y), the backward
    # through the batched entry point with one vector and without dvals (its
    # dxval pass walks only the vector's columns)
    h.allocPreBuffer()
    per = [(xk[xptr[v]:xptr[v + 1]], xv[xptr[v]:xptr[v + 1]], int(xptr[v + 1] - xptr[v]),
            t(np.array([0, xptr[v + 1] - xptr[v]], np.int32)), dY[:, v].contiguous())
           for v in range(nvec)]
    y1 = torch.empty(m, device=dev)
    with torch.cuda.stream(s):
        def plain():
            for v, (k1, v1, n1, p1, dy1) in enumerate(per):
                h.set_sparse_x(k1, v1, n1)
                h.run_adaptive(1.0, y1)
                h.spmspv_batched_backward(p1, k1, v1, 1.0, dy1, dxval[xptr[v]:xptr[v + 1]], None,
                                          x_total=n1)
        plain()
        tp = []
        for _ in range(max(2, reps // 3)):
            ev0.record(s)
            plain()
            ev1.record(s)
            s.synchronize()
            tp.append(ev0.elapsed_time(ev1))
    h.check_device_error()
    del g
    h.set_stream(stream)
    mb, mp = statistics.median(tb), statistics.median(tp)
    xn = int(xptr[-1])
    # compulsory bytes: the batch, A once per pass, the dense Y / dY once
    fwd_b = 12 * xn + 4 * (m + 1) + 8 * A.nnz + 4 * nvec * m
    bwd_b = 12 * xn + 2 * (4 * (m + 1) + 8 * A.nnz) + 4 * nvec * m + 4 * A.nnz + 4 * xn
    h.Destroy()
    return {"matrix": "chung-lu n %s, exponent 2.1, average degree 32, seed 5" % format(m, ","),
            "nnz": int(A.nnz), "nvec": nvec, "x_nnz_total": xn, "products": bins,
            "graph_fwd_bwd_ms": mb, "plain256_fwd_bwd_ms": mp, "speedup": mp / mb,
            "eff_gbs": (fwd_b + bwd_b) / (mb * 1e-3) / 1e9, "forward_within_1e-5": bool(ok),
            "backward_within_1e-5": bwd_ok,
            "options": "backward reuses the forward's inversion; dxval accumulated in the dvals pass "
                       "(atomic adds, not bitwise reproducible)",
            "note": "single calls: adaptive single-vector SpMSpV forward + one-vector backward "
                    "without dvals (less work than the batch, which also computes dvals)"}


def run_adjoint(torch, dev, stream, args):
    """Differentiable SpMV: the 5-point Laplacian on a 2048 x 2048 grid
    (4,194,304 rows, off-diagonals -1 + N(0, 0.01^2), seed 4), x and dy
    N(0,1).  Forward = the faster of the autotuned load-balanced SpMV and the
    naive CSR kernel; backward with dense dy = dx = A^T dy as a gather over
    the handle's CSC plus dvals on the pattern over the CSR (no atomics), and
    with dy masked to 1 % of the rows (sparse dy).  L2 flushed before every
    timed call."""
    import spmx
    from spmx import gen
    A = gen.laplacian(2048, 0.01, seed=4)
    m, n = A.m, A.n
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)  # noqa: E731
    h = spmx.SpmspvHandle(m, n, A.nnz, stream=stream)
    h.InputCSR(A.nnz, t(A.rowptr), t(A.col), t(A.val))
    h.ToCSC()
    h.holaPreprocess()
    backend = SPMV_BACKENDS.get(h.autotune(), "?")
    rng = np.random.default_rng(4)
    x = t(rng.standard_normal(n).astype(np.float32))
    dy = t(rng.standard_normal(m).astype(np.float32))
    k = m // 100
    key = np.sort(rng.choice(m, k, replace=False)).astype(np.int32)
    dk, dv = t(key), t(rng.standard_normal(k).astype(np.float32))
    h.set_x(x)
    y = torch.empty(m, device=dev)
    dx = torch.empty(n, device=dev)
    dvals = torch.empty(A.nnz, device=dev)
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=dev)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)

    def timed(fn):
        ts = []
        for it in range(3 + max(args.steps, 5)):
            flush.fill_(float(it))
            e0.record(stream)
            fn()
            e1.record(stream)
            stream.synchronize()
            if it >= 3:
                ts.append(e0.elapsed_time(e1))
        return statistics.median(ts)

    # the forward is the faster of the load-balanced back-end and the naive
    # CSR kernel (the banded Laplacian favours the latter)
    f_lb = timed(lambda: h.spmv(1.0, y))
    f_nv = timed(lambda: h.naivespmv(1.0, y))
    f_ms = min(f_lb, f_nv)
    if f_nv < f_lb:
        backend = "naive"
    b_ms = timed(lambda: h.spmv_backward(x, dy, dx, dvals))
    s_ms = timed(lambda: h.spmv_backward_sparse(x, dk, dv, k, dx, dvals))
    h.check_device_error()
    h.Destroy()
    fb = spmv_bytes(m, n, A.nnz)
    # dx pass: colptr, CSC rows + values, dy, dx; dvals pass: rowptr, columns, x, dy, dvals
    bb = (4 * (n + 1) + 8 * A.nnz + 4 * m + 4 * n) + (4 * (m + 1) + 4 * A.nnz + 4 * n + 4 * m + 4 * A.nnz)
    return {"matrix": "5-point Laplacian 2048^2, nnz %d, off-diagonals -1 + N(0, 0.01^2)" % A.nnz,
            "forward_backend": backend, "forward_ms": f_ms, "backward_dense_dy_ms": b_ms,
            "backward_sparse_dy_1pct_ms": s_ms, "backward_over_forward": b_ms / f_ms,
            "forward_gbs": fb / (f_ms * 1e-3) / 1e9, "backward_gbs": bb / (b_ms * 1e-3) / 1e9}


def run_powerlaw(torch, dev, stream, args):
    """SpMV on power-law matrices through the autotuned dispatcher: the
    Chung-Lu graph of the batched benchmark at 1,048,576 vertices (exponent
    2.1, average degree 32, N(0,1) values, seed 5) and R-MAT scale 20 (edge
    factor 16, seed 1, U(-1,1) values).  L2 flushed before every timed call;
    the roofline is the SpMV's compulsory bytes over the measured HBM peak;
    the result is checked against the FP64 oracle."""
    import spmx
    from spmx import gen
    import oracle.oracle as orc
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=dev)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    peak, peak_kind = peaks()
    out = []
    g = gen.rmat(20, 16, seed=1)
    g.val = np.random.default_rng(7).uniform(-1, 1, g.nnz).astype(np.float32)
    for name, A in (("chung-lu-1M", gen.chung_lu(1 << 20, 2.1, 32.0, seed=5)), ("rmat-20", g)):
        t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)  # noqa: E731
        h = spmx.SpmspvHandle(A.m, A.n, A.nnz, stream=stream)
        h.InputCSR(A.nnz, t(A.rowptr), t(A.col), t(A.val))
        h.holaPreprocess()
        backend = SPMV_BACKENDS.get(h.autotune(), "?")
        x_h = np.random.default_rng(3).uniform(-1, 1, A.n).astype(np.float32)
        h.set_x(t(x_h))
        y = torch.empty(A.m, device=dev)
        ts = []
        for it in range(3 + max(args.steps, 5)):
            flush.fill_(float(it))
            e0.record(stream)
            h.spmv(1.0, y)
            e1.record(stream)
            stream.synchronize()
            if it >= 3:
                ts.append(e0.elapsed_time(e1))
        h.check_device_error()
        y64, mag = orc.spmv_f64(A.rowptr, A.col, A.val, x_h)
        ok = bool(orc.within_tol(y.cpu().numpy(), y64, mag, 1e-5)[0])
        ms = statistics.median(ts)
        b = spmv_bytes(A.m, A.n, A.nnz)
        h.Destroy()
        out.append({"matrix": name, "nnz": A.nnz, "backend": backend, "ms": ms,
                    "gbs": b / (ms * 1e-3) / 1e9, "frac": b / (ms * 1e-3) / 1e9 / peak,
                    "peak_kind": peak_kind, "within_1e-5": ok})
    return out


def _ref_host_lib():
    """The reference's host routines compiled from its sources (oracle/_ref),
    or None where they were not built."""
    import ctypes
    so = os.path.join(ROOT, "oracle", "_ref", "libref_host.so")
    if not os.path.exists(so):
        return None
    lib = ctypes.CDLL(so)
    lib.ref_read_mtx.argtypes = [ctypes.c_char_p] + [ctypes.c_void_p] * 6
    lib.ref_read_mtx.restype = None
    lib.ref_free.argtypes = [ctypes.c_void_p]
    return lib


def run_ingest(torch, dev, stream, args):
    """Matrix ingestion: the 1M-row Zipf matrix (16,777,216 entries, entries
    shuffled with seed 1) written once as a MatrixMarket file, then
      parse   spmx_mtx_read on all host threads (file -> COO),
      gpu     pinned host-to-device copy of the COO + spmx_input_coo (radix
              sort by column, then by row, row pointers) -> device CSR,
    against the reference's ReadMTX (fscanf + std::sort by (row, col), one
    thread) compiled from its sources, or the oracle's restatement of it
    where that library is absent, run once on the same file.  The device CSR
    is checked bit for bit against the generator's CSR."""
    import ctypes
    import tempfile
    import spmx
    from spmx import gen, io
    import oracle.oracle as orc
    A = gen.zipf_1m()
    row = np.repeat(np.arange(A.m, dtype=np.int32), np.diff(A.rowptr))
    p = np.random.default_rng(1).permutation(A.nnz)
    tmpdir = tempfile.mkdtemp(prefix="spmx_ingest_")
    path = os.path.join(tmpdir, "zipf1m.mtx")
    try:
        io.write_mtx(path, io.Coo(A.m, A.n, row[p], A.col[p], A.val[p]))
        fbytes = os.path.getsize(path)
        parse = []
        for _ in range(3):
            t0 = time.perf_counter()
            C = io.read_mtx(path)
            parse.append(time.perf_counter() - t0)
        parse_s = statistics.median(parse)
        pinned = [torch.from_numpy(a).pin_memory() for a in (C.row, C.col, C.val)]
        dbuf = [torch.empty(C.nnz, dtype=t.dtype, device=dev) for t in pinned]
        h = spmx.SpmspvHandle(A.m, A.n, A.nnz, stream=stream)
        e0, e1, e2 = (torch.cuda.Event(enable_timing=True) for _ in range(3))
        h2d, sort = [], []
        for it in range(3 + max(args.steps // 4, 3)):
            stream.synchronize()
            e0.record(stream)
            with torch.cuda.stream(stream):
                for d, t in zip(dbuf, pinned):
                    d.copy_(t, non_blocking=True)
            e1.record(stream)
            h.InputCOO(C.nnz, *dbuf)  # synchronous
            e2.record(stream)
            stream.synchronize()
            if it >= 3:
                h2d.append(e0.elapsed_time(e1))
                sort.append(e1.elapsed_time(e2))
        rp, cl, vl = h.get_csr()
        exact = bool(np.array_equal(rp.cpu().numpy(), A.rowptr) and
                     np.array_equal(cl.cpu().numpy(), A.col) and
                     np.array_equal(vl.cpu().numpy().view(np.uint32), A.val.view(np.uint32)))
        h.check_device_error()
        h.Destroy()
        h2d_ms, sort_ms = statistics.median(h2d), statistics.median(sort)
        ref = _ref_host_lib()
        t0 = time.perf_counter()
        if ref is not None:
            m_, n_, k_ = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
            ptrs = [ctypes.c_void_p() for _ in range(3)]
            ref.ref_read_mtx(os.fsencode(path), ctypes.byref(m_), ctypes.byref(n_), ctypes.byref(k_),
                             *[ctypes.byref(q) for q in ptrs])
            ref_s = time.perf_counter() - t0
            for q in ptrs:
                ref.ref_free(q)
            ref_kind = "reference"
        else:
            orc.mtx_read_sorted(path)
            ref_s = time.perf_counter() - t0
            ref_kind = "port"
    finally:
        if os.path.exists(path):
            os.remove(path)
        os.rmdir(tmpdir)
    nnz = A.nnz
    e2e_s = parse_s + (h2d_ms + sort_ms) * 1e-3
    # algorithmic bytes of COO -> CSR: read 12 B per entry, write 8 B per entry + rowptr
    alg = 20 * nnz + 4 * (A.m + 1)
    return {"matrix": "zipf-1M, %d entries, MatrixMarket real general, %.0f MB, entries shuffled"
                      % (nnz, fbytes / 1e6),
            "parse_s": parse_s, "parse_entries_per_s": nnz / parse_s,
            "parse_mb_per_s": fbytes / 1e6 / parse_s, "parse_threads": orc.raw.cpu_threads(),
            "h2d_ms": h2d_ms, "coo_to_csr_ms": sort_ms,
            "coo_to_csr_entries_per_s": nnz / (sort_ms * 1e-3),
            "coo_to_csr_alg_gbs": alg / (sort_ms * 1e-3) / 1e9,
            "file_to_device_csr_s": e2e_s, "csr_bit_exact": exact,
            "reference_readmtx_s": ref_s, "reference_kind": ref_kind,
            "reference_cores": 1,
            "speedup_file_to_csr_vs_reference": ref_s / e2e_s}


def run_hybrid(torch, dev, stream, args):
    """The hybrid CSR/CSC split as a candidate ninth kernel: on the Zipf
    matrix (1,048,576 rows) and the Chung-Lu graph (1,048,576 vertices,
    exponent 2.1, average degree 32), the split's CSR share and the time of
    y = A x through the split against the autotuned load-balanced SpMV and
    the naive CSR kernel.  L2 flushed before every timed call."""
    import spmx
    from spmx import gen
    import oracle.oracle as orc
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=dev)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)

    def timed(fn):
        ts = []
        for it in range(3 + max(args.steps, 5)):
            flush.fill_(float(it))
            e0.record(stream)
            fn()
            e1.record(stream)
            stream.synchronize()
            if it >= 3:
                ts.append(e0.elapsed_time(e1))
        return statistics.median(ts)

    out = []
    for name, A in (("zipf-1M", gen.zipf_1m()), ("chung-lu-1M", gen.chung_lu(1 << 20, 2.1, 32.0, seed=5))):
        t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)  # noqa: E731
        h = spmx.SpmspvHandle(A.m, A.n, A.nnz, stream=stream)
        h.InputCSR(A.nnz, t(A.rowptr), t(A.col), t(A.val))
        h.ToCSC()
        backend = SPMV_BACKENDS.get(h.autotune(), "?")
        t0 = time.perf_counter()
        h.hybridPreprocess()
        prep_s = time.perf_counter() - t0
        csr_nnz, csc_nnz = h.hybrid_info()
        x_h = np.random.default_rng(3).uniform(-1, 1, A.n).astype(np.float32)
        h.set_x(t(x_h))
        y = torch.empty(A.m, device=dev)
        hy = timed(lambda: h.hybridspmv(1.0, y))
        y64, mag = orc.spmv_f64(A.rowptr, A.col, A.val, x_h)
        ok = bool(orc.within_tol(y.cpu().numpy(), y64, mag, 1e-5)[0])
        lb = timed(lambda: h.spmv(1.0, y))
        nv = timed(lambda: h.naivespmv(1.0, y))
        h.check_device_error()
        h.Destroy()
        out.append({"matrix": name, "nnz": A.nnz, "csr_share": csr_nnz / max(A.nnz, 1),
                    "preprocess_s": prep_s, "hybrid_ms": hy, "lb_spmv_ms": lb, "lb_backend": backend,
                    "naive_spmv_ms": nv, "hybrid_over_best": hy / min(lb, nv), "within_1e-5": ok})
    return out


def cpu_baseline(A, xs, binl):
    """The reference's CPU path on one core over one sweep: its own
    serialspmv (dense x) and SpmSpvCSCHost (sparse x), compiled from its
    sources (oracle/_ref), or the oracle's restatements where those were not
    built."""
    import oracle.oracle as orc
    colptr, row, cval = A.to_csc()
    m, n, nnz = A.m, A.n, A.nnz
    y = np.zeros(m, np.float32)
    yk = np.zeros(m, np.int32)
    P = lambda a: a.ctypes.data  # noqa: E731
    dense = [orc.sparse2dense_bits(n, k, v)[0] for _, k, v in xs]
    libs = ref_host_libs()
    import ctypes
    ynnz = ctypes.c_int()
    best = None
    for _ in range(3):
        t = 0.0
        for (d, key, val), xd in zip(xs, dense):
            t0 = time.perf_counter()
            if libs is None:
                if d >= 1.0:
                    orc.raw.cpu_spmv_serial(m, P(A.rowptr), P(A.col), P(A.val), P(xd), P(y), 1.0)
                else:
                    orc.raw.cpu_spmspv_csc_serial(m, P(colptr), P(row), P(cval), len(key), P(key),
                                                  P(val), P(y))
            elif d >= 1.0:
                libs[0].ref_serialspmv(m, n, nnz, P(A.rowptr), P(A.col), P(A.val), P(xd), P(y), 1.0)
            else:
                libs[1].ref_spmspv_csc_host(m, n, nnz, P(row), P(colptr), P(cval), len(key), P(key),
                                            P(val), ctypes.byref(ynnz), P(yk), P(y))
            t += time.perf_counter() - t0
        best = t if best is None else min(best, t)
    tot = sum(eff_bytes(m, n, nnz, len(k), b) for (_, k, _), b in zip(xs, binl))
    if libs is None:
        kind, what = "port", "the oracle's restatements of SpmSpvCSCHost / serialspmv"
    else:
        kind, what = "reference", ("the reference's own SpmSpvCSCHost / serialspmv compiled from its "
                                   "sources (SpmSpvCSCHost reads x into an int, so with U(-1,1) values "
                                   "its products are 0; it still does the same loads, adds and output "
                                   "pass)")
    return {"value": tot / best / 1e9, "unit": "GB/s", "cores": 1, "cpu": cpu_model(), "kind": kind,
            "sample": "one full 6-density sweep (best of 3), single thread: " + what,
            "ms": best * 1e3}


ONLY = ("powerlaw", "hybrid", "ingest", "batched-spmspv", "adjoint", "hola-spmv", "csr5-spmv", "naive-spmv", "tiled-spmv", "round-spmv", "hola-spmspv", "csc-lb-atomic",
        "csc-naive-atomic", "csc-bucket", "csc-lb-sort", "bfs-rmat14", "bfs-batched", "compact", "compact-to-host")


def run_only(args):
    """One kernel on the benchmark workload, K+W launches, for profiling
    (e.g. under ncu -k <kernel>); prints the mean time of the last K."""
    import torch
    import spmx
    dev = torch.device("cuda", 0)
    stream = torch.cuda.current_stream(dev)
    if args.only == "bfs-rmat14":
        print(json.dumps(run_bfs_plain(torch, dev, stream, args)))
        return 0
    if args.only == "bfs-batched":
        print(json.dumps(run_bfs_batched(torch, dev, stream, args)))
        return 0
    if args.only == "batched-spmspv":
        print(json.dumps(run_batched_spmspv(torch, dev, stream, args)))
        return 0
    if args.only == "adjoint":
        print(json.dumps(run_adjoint(torch, dev, stream, args)))
        return 0
    if args.only == "ingest":
        print(json.dumps(run_ingest(torch, dev, stream, args)))
        return 0
    if args.only == "hybrid":
        print(json.dumps(run_hybrid(torch, dev, stream, args)))
        return 0
    if args.only == "powerlaw":
        print(json.dumps(run_powerlaw(torch, dev, stream, args)))
        return 0
    A, xs = make_inputs()
    if args.matrix != "zipf1m":
        # the same x densities on a power-law matrix (SpMV kernels profile the dense x)
        from spmx import gen
        if args.matrix == "chunglu1m":
            A = gen.chung_lu(1 << 20, 2.1, 32.0, seed=5)
        else:
            A = gen.rmat(20, 16, seed=1)
            A.val = np.random.default_rng(7).uniform(-1, 1, A.nnz).astype(np.float32)
        xs = [(dd, *gen.sparse_vector(A.n, gen.density_nnz(A.n, dd), dist="uniform",
                                       seed=1000 + gen.density_nnz(A.n, dd))) for dd in DENSITIES]
    d = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)  # noqa: E731
    rp, cl, vl = d(A.rowptr), d(A.col), d(A.val)
    h = spmx.SpmspvHandle(A.m, A.n, A.nnz, stream=stream)
    h.InputCSR(A.nnz, rp, cl, vl)
    h.ToCSC()
    h.holaPreprocess()
    h.CSR5Preprocess()
    h.tiledPreprocess()
    h.roundPreprocess(0, args.round_parts)
    h.allocPreBuffer()
    if args.col_lanes:
        h.set_naive_lanes(0, args.col_lanes)
    dens = 1.0 if args.only.endswith("spmv") else args.density
    k = [x for x in xs if abs(x[0] - dens) < 1e-12][0]
    kd, vd = d(k[1]), d(k[2])
    h.set_sparse_x(kd, vd, len(k[1]))
    h.sparse2bitarray()
    y = torch.empty(A.m, device=dev)
    yk = torch.empty(A.m, dtype=torch.int32, device=dev)
    yv = torch.empty(A.m, device=dev)
    if args.only.startswith("compact"):
        # the compaction of y = A x at the chosen density: to device buffers,
        # or straight into pinned host memory (the e2e path's read-back)
        from spmx import abi
        h.spmspv_csc(0, 0, 1.0, y, sync=False)
        hk = torch.empty(A.m, dtype=torch.int32).pin_memory()
        hv = torch.empty(A.m, dtype=torch.float32).pin_memory()
        hc = torch.zeros(1, dtype=torch.int32).pin_memory()

        def compact(to_host):
            rc = (abi.lib.spmx_dense2sparse_to_host(h._h, A.m, y.data_ptr(), hk.data_ptr(), hv.data_ptr(),
                                                     hc.data_ptr()) if to_host else
                  abi.lib.spmx_dense2sparse_outer(h._h, A.m, y.data_ptr(), None, yk.data_ptr(), yv.data_ptr()))
            if rc:
                raise RuntimeError(f"compaction failed: {rc}")
    run = {
        "compact": lambda: compact(False),
        "compact-to-host": lambda: compact(True),
        "hola-spmv": lambda: h.holaspmv(1.0, y),
        "csr5-spmv": lambda: h.csr5spmv(1.0, y),
        "naive-spmv": lambda: h.naivespmv(1.0, y),
        "tiled-spmv": lambda: h.tiledspmv(1.0, y),
        "round-spmv": lambda: h.roundspmv(1.0, y),
        "hola-spmspv": lambda: h.holaspmspv(1.0, y),
        "csc-lb-atomic": lambda: h.spmspv_csc(1, 0, 1.0, y, sync=False),
        "csc-naive-atomic": lambda: h.spmspv_csc(0, 0, 1.0, y, sync=False),
        "csc-bucket": lambda: h.CscBasedBucketSpmspv(1.0, y, yk, yv),
        "csc-lb-sort": lambda: h.spmspv_csc(1, 1, 1.0, None, yk, yv),
    }[args.only]
    s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ts = []
    for it in range(args.warmup + args.steps):
        s.record(stream)
        run()
        e.record(stream)
        stream.synchronize()
        if it >= args.warmup:
            ts.append(s.elapsed_time(e))
    h.check_device_error()
    out = {"only": args.only, "density": dens, "ms": statistics.mean(ts), "min_ms": min(ts)}
    if args.only.startswith("tiled"):
        out["tiled"] = h.tiled_info()
    if args.only.startswith("round"):
        out["round"] = h.round_info()
    print(json.dumps(out))
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-bfs", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-batched", action="store_true")
    ap.add_argument("--no-ingest", action="store_true")
    ap.add_argument("--no-ref-gpu", action="store_true",
                    help="with --impl reference: leave out the reference's own GPU kernels, rebuilt "
                         "for sm_100a, on the same sweep (timed by default)")
    ap.add_argument("--tune-cache", default=None,
                    help="autotuner cache file: a second run with the same file (e.g. under a profiler, "
                         "whose serialised timings would mislead the tuner) reuses the first run's choices")
    ap.add_argument("--only", choices=ONLY, help="run one kernel (profiling helper)")
    ap.add_argument("--density", type=float, default=0.1)
    ap.add_argument("--col-lanes", type=int, default=0,
                    help="with --only: lanes per x entry of the naive CSC scatter (0: from the mean column length)")
    ap.add_argument("--round-parts", type=int, default=1, choices=[1, 2, 4],
                    help="--only round-spmv: CTAs per row block of the round format")
    ap.add_argument("--batched-log2n", type=int, default=22,
                    help="log2 of the Chung-Lu size of the batched SpMSpV line (22 = the benchmark's; "
                         "smaller for profiling)")
    ap.add_argument("--matrix", default="zipf1m", choices=["zipf1m", "chunglu1m", "rmat20"],
                    help="with --only: the matrix (the benchmark's Zipf matrix by default)")
    args = ap.parse_args()
    if args.only:
        return run_only(args)
    world, rank, local = dist_init(args)
    try:
        if args.impl == "reference":
            rc = run_reference(args, world, rank)
        else:
            rc = run_ours(args, world, rank, local)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()
    return rc


if __name__ == "__main__":
    sys.exit(main())
