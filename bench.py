"""Fock-build throughput of QUICK's direct-SCF two-electron path on B200.

One step = one two-electron Fock build G(D) of the workload molecule
(QUICK's gpu_get2e_: screening, all angular classes, O + G), inputs resident
in HBM.  Metric: shell quartets per second, a shell quartet being one
(IJ|KL) block of unique integrals over angular sub-shells that passes QUICK's
Schwarz and density screens.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--part all|fock|xc|scf|batch]

The default workload is (H2O)32 in 6-31G** (800 Cartesian basis functions),
seeded geometry, CUTOFF=1e-10 semantics (integral cutoff 1e-10, primitive
limit 1e-20).  For N > 1 every rank builds the Fock matrix of its own replica
(weak scaling, no collective on the data path); the time is the max over ranks.

The one JSON line also carries: the same build end to end through the host
entry points (e2e), replayed from a CUDA graph, and with the mixed FP32/FP64
split; the two-electron gradient; the XC quadrature (xc); SCF + gradient
seconds per molecule, all-FP64 and mixed, with full and delta-D Fock builds,
plus a Kohn-Sham and a cc-pVTZ case (scf); molecules per second for many
small clusters (batch); the CPU baseline, QUICK's own kernel compiled for
the host cores; and reference_gpu, QUICK's own CUDA built for sm_100a and
run on the same GPU on the same workload (in a process of its own).
"""
import argparse
import gc
import json
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

# pure-Python input builders (no library load): QUICK's basis arrays, the
# seeded molecules, the model density and QUICK's density screen
from quick_b200.molecule import model_density  # noqa: E402
from quick_b200.scf import shell_cut_matrix  # noqa: E402

WORKLOAD = dict(name="(H2O)32 6-31G** RHF Fock build", grid=(4, 4, 2), basis="6-31G**", seed=0,
                integral_cutoff=1e-10, prim_limit=1e-20)
# mixed-precision split: shell quartets whose Y_ab Y_cd DNMax bound is below this run in FP32
# DRAM bytes (read + write) of the class kernels of one FP64 build of the
# workload, from one ncu capture (cold caches): the roofline's traffic
FOCK_BUILD_DRAM_BYTES = 24.8e9
MIXED_CUT = 1e-3


class Clocks:
    """nvidia-smi sampling during the timed region."""

    def __init__(self, index):
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(index), "--query-gpu=" + q,
                                       "--format=csv,noheader,nounits", "-lms", "200"],
                                      stdout=self.f, stderr=subprocess.DEVNULL)
        except FileNotFoundError:
            self.p = None

    def stop(self):
        if self.p is None:
            return None
        self.p.terminate()
        self.p.wait()
        rows = []
        with open(self.f.name) as fh:
            for ln in fh:
                t = [x.strip() for x in ln.split(",")]
                if len(t) >= 9:
                    rows.append(t)
        os.unlink(self.f.name)
        if not rows:
            return None
        num = lambda s: s.replace(".", "", 1).isdigit()
        sm = [float(r[1]) for r in rows if num(r[1])]
        mx = [float(r[2]) for r in rows if num(r[2])]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({n for r in rows for n, v in zip(names, r[5:9]) if v.lower() == "active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


def dist_setup():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if ws > 1:
        import datetime
        import torch
        import torch.distributed as dist
        os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
        # NCCL between the GPUs; gloo where there are none (the CPU tests of
        # this rank logic)
        backend = "nccl" if torch.cuda.is_available() else "gloo"
        if backend == "nccl":
            torch.cuda.set_device(local)
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=300))
    return ws, rank, local


def barrier(ws):
    if ws > 1:
        import torch.distributed as dist
        dist.barrier()


def max_over_ranks(x, ws):
    if ws == 1:
        return x
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def batch_sizes(nmol, rank):
    """Cluster sizes n (uniform in 1..12) of one rank's molecules in the
    batch line: seeded by rank, so every rank runs its own list."""
    return np.random.default_rng(1234 + rank).integers(1, 13, size=nmol)


WARMUP_SAMPLE = dict(name="(H2O)4 6-31G* RHF Fock build", grid=(2, 2, 1), basis="6-31G*")


def workload_config(nbasis, quartets):
    """The config object of the Fock-build line, the same for both arms."""
    return {"workload": WORKLOAD["name"], "nbasis": nbasis, "quartets_per_step": quartets,
            "integral_cutoff": WORKLOAD["integral_cutoff"], "prim_limit": WORKLOAD["prim_limit"],
            "method": "HF (full exchange)", "density": "model density, seed %d" % WORKLOAD["seed"],
            "l2": "GPU arm: flushed (256 MB write) before every timed step; host arm: not applicable",
            "parallelism": "replicas"}


def cpu_reference(threads, steps=1, warmup=0):
    """QUICK's own two-electron kernel (src/cuda/gpu_get2e_subs.h, driven by
    QUICK's src/cuda/gpu.cu bridge) compiled for the host cores
    (oracle/_ref/libquickref.so), timed on the workload itself: one step is
    one full Fock build of (H2O)32 in 6-31G** through QUICK's gpu_upload_* /
    gpu_get2e_ sequence.  Warm-up steps run the same kernel on (H2O)4 in
    6-31G*.  The shell quartets per step are counted by QUICK's own walk
    (oracle.ref_quartet_counts: once per unordered pair of shell pairs, the
    count the GPU arm reports; tests/test_gpu_configs.py holds the two equal).
    Nothing of this package's library is loaded.
    Returns (quartets/s, quartets per step, s per step, raw iclass calls)."""
    import oracle
    from quick_b200.basis import build_basis
    from quick_b200.molecule import water_cluster
    cut, plim = WORKLOAD["integral_cutoff"], WORKLOAD["prim_limit"]

    def setup(grid, basis):
        m = water_cluster(grid, seed=WORKLOAD["seed"])
        b = build_basis(m.symbols, basis)
        Y, cp = oracle.schwarz(b, m.xyz_bohr)
        keep = oracle.ref_upload_molecule(m, b, Y, cp, threads=threads)
        D = model_density(m, b, seed=WORKLOAD["seed"])
        return b, keep, D, shell_cut_matrix(b, D)

    if warmup:
        b, keep, D, cm = setup(WARMUP_SAMPLE["grid"], WARMUP_SAMPLE["basis"])
        for _ in range(warmup):
            oracle.ref_get2e(np.zeros_like(D), D, cm, cut, plim)
    b, keep, D, cm = setup(WORKLOAD["grid"], WORKLOAD["basis"])
    ts, counts = [], set()
    for _ in range(steps):
        t0 = time.perf_counter()
        oracle.ref_get2e(np.zeros_like(D), D, cm, cut, plim)
        ts.append(time.perf_counter() - t0)
        counts.add(oracle.ref_quartet_counts())
    assert len(counts) == 1, counts
    raw, nq = counts.pop()
    return nq / np.mean(ts), nq, float(np.mean(ts)), raw


def gpu_reference(steps, warmup, device=0):
    """QUICK's own GPU path on this GPU: src/cuda/gpu.cu, gpu_type.cu,
    gpu_get2e.cu and gpu_getxc.cu built unchanged by nvcc for sm_100a with
    QUICK's flags and configuration (oracle/_ref/gpu, build_ref.py --gpu),
    driven through QUICK's gpu_init_ / gpu_upload_* / gpu_get2e_ sequence on
    the same (H2O)32 workload.  A step is QUICK's per-iteration sequence
    (src/hfoperator.f90:76-98): gpu_upload_method_, gpu_upload_calculated_
    (host O and D), gpu_upload_cutoff_ (cutMatrix), gpu_get2e_ (its kernel,
    the download of the fixed-point O and the conversion on the host),
    timed by wall clock (the bridge returns only after its download); the
    kernel's own time is QUICK's CUDA-event timer around its launch.  The
    shell-quartet count is QUICK's own walk on the same inputs (the config-1
    fixture, counted by QUICK's kernel on the host).  Warm-up steps run the
    same workload.  Loads nothing from quick_b200's library."""
    import oracle
    from quick_b200.basis import build_basis
    from quick_b200.molecule import water_cluster
    cut, plim = WORKLOAD["integral_cutoff"], WORKLOAD["prim_limit"]
    m = water_cluster(WORKLOAD["grid"], seed=WORKLOAD["seed"])
    b = build_basis(m.symbols, WORKLOAD["basis"])
    Y, cp = oracle.schwarz(b, m.xyz_bohr)
    keep = oracle.ref_upload_molecule(m, b, Y, cp, spdf="gpu", device=device)  # noqa: F841
    D = model_density(m, b, seed=WORKLOAD["seed"])
    cm = shell_cut_matrix(b, D)
    for _ in range(warmup):
        oracle.ref_get2e_gpu_timed(np.zeros_like(D), D, cm, cut, plim)
    walls, kerns = [], []
    for _ in range(steps):
        O, wall, kern = oracle.ref_get2e_gpu_timed(np.zeros_like(D), D, cm, cut, plim)
        walls.append(wall)
        kerns.append(kern)
    z = np.load(os.path.join(ROOT, "tests", "golden", "config1_water32_631gss.npz"))
    full = WORKLOAD["grid"] == (4, 4, 2) and WORKLOAD["basis"] == "6-31G**"
    nq = int(z["unique_quartets"]) if full else None     # QUICK's own count of this workload
    par = (quick_parity(np.ascontiguousarray(O.T), nq, b.nbasis) or {}) if full else {}
    wall, kern = float(np.mean(walls)), float(np.mean(kerns))
    # QUICK's two-electron gradient (src/gradient.f90:279-286) on the same
    # density: one warm-up call, one timed (each takes seconds)
    gw, gk = [], []
    for i in range(2):
        g, w, k = oracle.ref_grad_gpu_timed(3 * m.natom, D, cm, cut, plim)
        if i:
            gw.append(w)
            gk.append(k)
    # QUICK's B3LYP XC quadrature on its SG1 grid (gpu_getxc_), the density of the xc line
    from quick_b200.basis import sigrad2
    rng = np.random.default_rng(WORKLOAD["seed"])
    Cx = rng.standard_normal((b.nbasis, m.n_electrons // 2)) * 0.05
    Dx = np.asfortranarray(2.0 * Cx @ Cx.T)
    xw = []
    for i in range(2):
        _, exc, nel, w = oracle.ref_getxc_gpu_timed(Dx, sigrad2(b), method=1)
        if i:
            xw.append(w)
    if not full:
        return {"workload": WORKLOAD["name"], "ms_per_step": wall * 1e3, "kernel_ms": kern,
                "gradient_kernel_ms": float(np.mean(gk)), "xc_ms_per_call": float(np.mean(xw)) * 1e3}
    return {"value": nq / wall, "unit": "quartets/s", "ms_per_step": wall * 1e3,
            "kernel_ms": kern, "kernel_quartets_per_s": nq / (kern * 1e-3), "quartets_per_step": nq,
            "steps": steps, "warmup": warmup,
            "max_abs_dF_vs_quick_host_sampled": par.get("max_abs_dF_sampled"),
            "gradient": {"ms_per_call": float(np.mean(gw)) * 1e3, "kernel_ms": float(np.mean(gk)),
                         "max_abs_dg_vs_quick_host": float(np.abs(g - z["grad"]).max()), "calls": len(gw),
                         "what": "gpu_upload_calculated_/gpu_upload_cutoff_/gpu_upload_grad_/gpu_grad_ wall time; "
                                 "kernel_ms: QUICK's event timers around its gradient launches, summed"},
            "xc": {"ms_per_call": float(np.mean(xw)) * 1e3, "exc": exc, "electrons": nel, "calls": len(xw),
                   "what": "B3LYP, QUICK's SG1 grid: gpu_upload_method_/gpu_upload_calculated_/gpu_getxc_ wall "
                           "time (its kernel launch has no event timer)"},
            "what": "QUICK's own CUDA (gpu.cu bridge + get2e_kernel, spd build, -O3 -use_fast_math, QUICK's "
                    "config.cuda.h) built unchanged for sm_100a and run on this GPU on %s; value: the whole "
                    "gpu_upload_calculated_/gpu_upload_cutoff_/gpu_get2e_ sequence from host buffers (its e2e), "
                    "kernel_ms: QUICK's own CUDA-event timer around get2e_kernel" % WORKLOAD["name"]}


def quick_parity(G, quartets, n):
    """max |G - G_QUICK| over the fixture's 20000 sampled elements and the
    diagonal, the largest projection error, and whether the shell-quartet
    count equals QUICK's (tests/golden/config1_water32_631gss.npz: QUICK's
    kernel compiled for the host on this workload and density).  G is
    row-major here; it is symmetric."""
    path = os.path.join(ROOT, "tests", "golden", "config1_water32_631gss.npz")
    if not os.path.exists(path) or WORKLOAD["grid"] != (4, 4, 2) or WORKLOAD["basis"] != "6-31G**":
        return None
    z = np.load(path)
    if int(z["nbasis"]) != n:
        return None
    rng = np.random.default_rng(123)           # the fixture's probes (make_config_golden.probes)
    R = rng.standard_normal((n, 8))
    idx = rng.integers(0, n, size=(20000, 2))
    return {"max_abs_dF_sampled": float(max(np.abs(G[idx[:, 0], idx[:, 1]] - z["sample"]).max(),
                                            np.abs(np.diag(G) - z["diag"]).max())),
            "max_abs_dGR": float(np.abs(G @ R - z["GR"]).max()),
            "quartets_equal_quick": int(z["unique_quartets"]) == int(quartets),
            "quick_unique_quartets": int(z["unique_quartets"]),
            "reference": "QUICK's get2e kernel compiled for the host, same inputs (20000 sampled elements, "
                         "the diagonal and 8 projections of the 800 x 800 matrix)"}


def run_ours(args, ws, rank, local):
    import torch
    from quick_b200 import capi, flops
    from quick_b200.basis import build_basis
    from quick_b200.molecule import water_cluster

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    # one non-default stream for the library and every timed event: the
    # device-side Fock build is asynchronous on the library stream
    stream = torch.cuda.Stream(dev)
    torch.cuda.set_stream(stream)
    m = water_cluster(WORKLOAD["grid"], seed=WORKLOAD["seed"])
    b = build_basis(m.symbols, WORKLOAD["basis"])
    n = b.nbasis
    sess = capi.Session(local)
    lib = capi.lib()
    lib.qb_set_stream(capi.C.c_void_p(stream.cuda_stream))
    sess.upload_molecule(m, b)          # Schwarz bounds from the GPU kernel
    D = model_density(m, b, seed=WORKLOAD["seed"])
    cm = shell_cut_matrix(b, D)
    cutoff, plim = WORKLOAD["integral_cutoff"], WORKLOAD["prim_limit"]
    O0 = np.zeros((n, n), order="F")
    sess.get2e(O0, D, cm, cutoff, plim, method=0)    # uploads cutoffs, sizes the quartet lists
    dD = torch.from_numpy(np.ascontiguousarray(D)).to(dev)
    dO = torch.zeros((n, n), dtype=torch.float64, device=dev)
    dOut = torch.empty_like(dO)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)   # > 126 MB L2

    def step():
        rc = lib.qb_fock_device(capi.C.c_void_p(dD.data_ptr()), capi.C.c_void_p(dO.data_ptr()),
                                capi.C.c_void_p(dOut.data_ptr()))
        if rc:
            capi.check()

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    # lanes per quartet of each class autotuned on this build's quartet lists
    # (qb_autotune_classes), then warmed up again
    groups64 = sess.autotune()
    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    quartets = sess.fock_stats()["quartets"]
    ncls = capi.C.c_int(0)
    cl = np.zeros(4 * 128, dtype=np.int32)
    cq = np.zeros(128, dtype=np.int64)
    lib.qb_class_info(capi.C.byref(ncls), capi._ptr(cl), capi._ptr(cq), 128)
    npq = np.zeros(128, dtype=np.int64)
    lib.qb_count_prim_quartets(capi._ptr(npq), 128)
    capi.check()
    k = ncls.value
    # per class the smaller of the generator-graph and the definition count
    alg_flops = flops.fock_flops(cl[:4 * k].reshape(k, 4), cq[:k], npq[:k], exchange=True, table="min")
    alg_flops_tables = {t: flops.fock_flops(cl[:4 * k].reshape(k, 4), cq[:k], npq[:k], exchange=True, table=t)
                        for t in ("generator", "definition")}
    peak64 = capi.C.c_double(0)
    lib.qb_fma_peak(1, capi.C.byref(peak64))

    barrier(ws)
    torch.cuda.synchronize()
    clocks = Clocks(local) if rank == 0 else None
    l0 = lib.qb_launch_count()
    e0 = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    e1 = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    eri_ms, scr_ms = [], []
    for i in range(args.steps):
        flush.zero_()
        e0[i].record(stream)
        step()
        e1[i].record(stream)
        s = sess.fock_stats()
        eri_ms.append(s["ms_eri"])
        scr_ms.append(s["ms_screen"])
    torch.cuda.synchronize()
    barrier(ws)
    launches = lib.qb_launch_count() - l0
    step_ms = [a.elapsed_time(b_) for a, b_ in zip(e0, e1)]
    ms = max_over_ranks(float(np.mean(step_ms)), ws)
    clk = clocks.stop() if clocks else None

    # the timed step's result against QUICK's own kernel on the same inputs
    # (fixture of tests/golden/make_config_golden.py), outside the timed region
    parity = quick_parity(dOut.double().cpu().numpy(), quartets, n)

    # end to end through QUICK's C ABI with pinned host buffers: upload D, O and
    # cutMatrix, Fock build, download O, every step
    pinD = torch.from_numpy(np.asfortranarray(D).ravel(order="F").copy()).pin_memory()
    pinO = torch.zeros(n * n, dtype=torch.float64).pin_memory()
    pinCM = torch.from_numpy(np.asfortranarray(cm).ravel(order="F").copy()).pin_memory()
    ptr = lambda t: capi.C.c_void_p(t.data_ptr())
    one = capi.C.byref
    co = torch.zeros(1, dtype=torch.float64)
    ec0, ec1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    barrier(ws)
    torch.cuda.synchronize()
    ec0.record(stream)
    for i in range(args.steps):
        pinO.zero_()
        lib.gpu_upload_method_(one(capi.C.c_int(0)))
        lib.gpu_upload_calculated_(ptr(pinO), ptr(co), ptr(co), ptr(pinD))
        lib.gpu_upload_cutoff_(ptr(pinCM), one(capi.C.c_double(cutoff)), one(capi.C.c_double(plim)), None)
        lib.gpu_get2e_(ptr(pinO))
    ec1.record(stream)
    torch.cuda.synchronize()
    capi.check()
    e2e_ms = max_over_ranks(ec0.elapsed_time(ec1) / args.steps, ws)

    # the same step replayed from a CUDA graph (qb_fock_device allocates and
    # waits for nothing after the warm-up, so one capture holds the build)
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(graph, stream=stream):
        step()
    torch.cuda.synchronize()
    g0 = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    g1 = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    for i in range(args.steps):
        flush.zero_()
        g0[i].record(stream)
        graph.replay()
        g1[i].record(stream)
    torch.cuda.synchronize()
    graph_ms = max_over_ranks(float(np.mean([a.elapsed_time(c) for a, c in zip(g0, g1)])), ws)
    del graph

    # mixed precision: quartets with Y_ab Y_cd DNMax < MIXED_CUT in FP32, same
    # density; error against this FP64 build
    G64 = dOut.double().cpu().numpy().copy()
    lib.qb_set_mixed_precision(capi.C.c_double(MIXED_CUT))
    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    groups32 = sess.autotune()   # lanes per quartet of the FP32 class kernels, on this build's FP32 lists
    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    barrier(ws)
    m0 = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    m1 = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    mix_eri = []
    for i in range(args.steps):
        flush.zero_()
        m0[i].record(stream)
        step()
        m1[i].record(stream)
        mix_eri.append(sess.fock_stats()["ms_eri"])
    torch.cuda.synchronize()
    barrier(ws)
    mix_ms = max_over_ranks(float(np.mean([a.elapsed_time(c) for a, c in zip(m0, m1)])), ws)
    split = sess.fock_split()
    Gmx = dOut.double().cpu().numpy()
    lib.qb_set_mixed_precision(capi.C.c_double(0.0))
    Dn = np.ascontiguousarray(D)
    mixed = {"value": quartets * ws / (mix_ms * 1e-3), "unit": "quartets/s", "ms_per_step": mix_ms,
             "kernel_ms": float(np.mean(mix_eri)), "cut": MIXED_CUT,
             "fp32_quartet_fraction": split["fp32"] / max(1, split["fp32"] + split["fp64"]),
             "speedup_vs_fp64": ms / mix_ms,
             "abs_dE2_vs_fp64_Eh": float(abs(0.5 * np.sum(Dn * (Gmx - G64)))),
             "max_abs_dF_vs_fp64": float(np.abs(Gmx - G64).max())}

    # the two-electron gradient of the same density through gpu_grad_
    # (QUICK's gradient call sequence, host buffers)
    g_in = np.zeros(3 * m.natom)
    for _ in range(args.warmup):
        sess.grad(g_in, D, cm, cutoff, plim)
    ggroups64 = sess.autotune_grad()   # lanes per quartet of the light gradient classes
    for _ in range(args.warmup):
        sess.grad(g_in, D, cm, cutoff, plim)
    gr_ms, gr_e2e = [], []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        sess.grad(g_in, D, cm, cutoff, plim)
        gr_e2e.append(1e3 * (time.perf_counter() - t0))
        gr_ms.append(sess.grad_stats()["ms"])
    gq = sess.grad_stats()["quartets"]
    g64 = sess.grad(g_in, D, cm, cutoff, plim)
    # the same gradient with the mixed split
    lib.qb_set_mixed_precision(capi.C.c_double(MIXED_CUT))
    for _ in range(args.warmup):
        sess.grad(g_in, D, cm, cutoff, plim)
    ggroups32 = sess.autotune_grad()
    for _ in range(args.warmup):
        sess.grad(g_in, D, cm, cutoff, plim)
    grm_ms = []
    for _ in range(args.steps):
        gmx = sess.grad(g_in, D, cm, cutoff, plim)
        grm_ms.append(sess.grad_stats()["ms"])
    lib.qb_set_mixed_precision(capi.C.c_double(0.0))
    grm = max_over_ranks(float(np.mean(grm_ms)), ws)
    light = [i for i in range(k) if cq[i] > 0 and sum(cl[4 * i:4 * i + 4]) <= 2]
    grad_line = {"metric": "two-electron gradient shell quartets/s (FP64)", "quartets_per_call": gq,
                 "lane_groups": {"fp64": {"%d%d%d%d" % tuple(cl[4 * i:4 * i + 4]): int(ggroups64[i]) for i in light},
                                 "fp32": {"%d%d%d%d" % tuple(cl[4 * i:4 * i + 4]): int(ggroups32[i]) for i in light}},
                 "kernel_ms": max_over_ranks(float(np.mean(gr_ms)), ws),
                 "value": gq * ws / (max_over_ranks(float(np.mean(gr_ms)), ws) * 1e-3), "unit": "quartets/s",
                 "e2e_ms_per_call": max_over_ranks(float(np.mean(gr_e2e)), ws),
                 "mixed": {"kernel_ms": grm, "value": gq * ws / (grm * 1e-3), "cut": MIXED_CUT,
                           "speedup_vs_fp64": max_over_ranks(float(np.mean(gr_ms)), ws) / grm,
                           "max_abs_dgrad_vs_fp64": float(np.abs(gmx - g64).max())},
                 "note": "gpu_upload_calculated_/cutoff_/grad_ + gpu_grad_ per call; e2e by host clock"}

    mean_eri = float(np.mean(eri_ms))
    achieved = alg_flops / (mean_eri * 1e-3) / 1e12
    peak = peak64.value / 1e3
    out = {
        "metric": "Fock-build shell quartets/s (FP64)",
        "value": quartets * ws / (ms * 1e-3),
        "unit": "quartets/s",
        "n_gpus": ws,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": ms,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64",
        "data": "synthetic: seeded (H2O)32 geometry, model density",
        "config": workload_config(n, quartets),
        "lane_groups": {"note": "lanes per quartet, autotuned per class (qb_autotune_classes)",
                        "fp64": {"%d%d%d%d" % tuple(cl[4 * i:4 * i + 4]): int(groups64[i])
                                 for i in range(k) if cq[i] > 0 and sum(cl[4 * i:4 * i + 4]) < 6},
                        "fp32": {"%d%d%d%d" % tuple(cl[4 * i:4 * i + 4]): int(groups32[i])
                                 for i in range(k) if cq[i] > 0 and sum(cl[4 * i:4 * i + 4]) < 6}},
        "parity_vs_quick": parity,
        "e2e": {"value": quartets * ws / (e2e_ms * 1e-3), "unit": "quartets/s",
                "h2d_bytes_per_step": int(2 * n * n * 8 + b.nshell ** 2 * 8),
                "d2h_bytes_per_step": int(n * n * 8), "ms_per_step": e2e_ms},
        "roofline": {"bound": "fp64", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                     "frac": achieved / peak if peak else None, "traffic": FOCK_BUILD_DRAM_BYTES,
                     "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum summed over the class "
                                       "kernels of one FP64 build (cold caches), "
                                       "profiles/fock_class_kernels_water32_631gss.md",
                     "kernel": "fock_class_kernel<LA,LB,LC,LD> (all classes of one build)",
                     "peak_source": "measured: FP64 FMA-chain probe run in this process (qb_fma_peak)",
                     "flops_per_step": alg_flops,
                     "flops_per_step_by_table": alg_flops_tables,
                     "flops_note": "per class the smaller of two counts, both from the recurrences and not from "
                                   "the kernels: the generator's dependency graph and the recurrence definitions "
                                   "(quick_b200/flops.py definition_class)",
                     "kernel_ms": mean_eri,
                     "screen_ms": float(np.mean(scr_ms))},
        "gpu_launches": int(launches),
        "cuda_graph": {"ms_per_step": graph_ms, "value": quartets * ws / (graph_ms * 1e-3), "unit": "quartets/s",
                       "note": "the same step captured once with torch.cuda.graph and replayed"},
        "mixed": mixed,
        "gradient": grad_line,
    }
    if clk:
        out["clocks"] = clk
    if args.classes:
        out["classes"] = {"%d%d%d%d" % tuple(cl[4 * i:4 * i + 4]): [int(cq[i]), int(npq[i])] for i in range(k)}
    return out


def measured_hbm_gbs():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as fh:
            return float(json.load(fh)["hbm_gbs"]), "measured (MEASURED_PEAKS.json hbm_gbs)"
    except Exception:
        return 6650.0, "fallback (6.65 TB/s)"


def run_scf(args, ws, rank, local):
    """SCF + gradient seconds per molecule for (H2O)32 in 6-31G** (RHF,
    integral cutoff 1e-10, density RMS 1e-8): the device-resident SCF from
    the SAD guess and the full analytic gradient, all-FP64 against the mixed
    FP32/FP64 split, each with full and with delta-D Fock builds.  Wall clock
    per molecule (host-driven loop with a convergence test every iteration),
    max over ranks; one untimed molecule first."""
    import torch
    from quick_b200 import scf
    from quick_b200.molecule import water_cluster
    from quick_b200 import capi
    torch.cuda.set_device(local)
    m = water_cluster(WORKLOAD["grid"], seed=WORKLOAD["seed"])
    # nine molecules per variant: host-side jitter on shared boxes makes one
    # or two molecules of a handful slow, and the median has to see past it
    nmol = max(1, min(args.steps, 9))
    # one session for every molecule (the library's tables and buffers are
    # reused); warm-up molecules, all-FP64 and mixed, each followed by the
    # lane-group autotuners of the Fock and gradient kernels (FP64, then FP32)
    sess = capi.Session(local)
    scf.run_rhf_device(m, WORKLOAD["basis"], 1e-10, 1e-20, conv=1e-8, device=local, session=sess)
    sess.autotune()
    sess.autotune_grad()
    scf.run_rhf_device(m, WORKLOAD["basis"], 1e-10, 1e-20, conv=1e-8, device=local, session=sess,
                       mixed_cut=MIXED_CUT)
    sess.autotune()
    sess.autotune_grad()
    res = {}
    # every variant but the first replays each SCF iteration from a CUDA graph
    for tag, kw in (("fp64_eager", {}), ("fp64", dict(graph=True)), ("mixed", dict(mixed_cut=MIXED_CUT, graph=True)),
                    ("fp64_delta_d", dict(incremental=True, graph=True)),
                    ("mixed_delta_d", dict(mixed_cut=MIXED_CUT, incremental=True, graph=True))):
        secs, runs = [], []
        for _ in range(nmol):
            # the previous molecule's objects (engines, graphs, device tensors)
            # are collected before this molecule's clock starts
            gc.collect()
            torch.cuda.synchronize()
            barrier(ws)
            r, g = scf.run_rhf_device(m, WORKLOAD["basis"], 1e-10, 1e-20, conv=1e-8, device=local, session=sess,
                                      **kw)
            secs.append(r.seconds)
            runs.append((r, g))
        phases_each = [dict({k: round(v, 3) for k, v in rr.timings.items() if k in ("setup", "scf", "gradient")},
                            slowest_iteration=round(max(h[2] for h in rr.history), 4)) for rr, _ in runs]
        r, g = runs[-1]
        res[tag] = dict(seconds_per_molecule=max_over_ranks(float(np.median(secs)), ws),
                        seconds_each=[round(x, 4) for x in secs], phases_each=phases_each,
                        seconds_min=min(secs),
                        molecules_per_s=ws / max_over_ranks(float(np.median(secs)), ws),
                        energy=r.energy, iterations=r.iterations, converged=bool(r.converged),
                        fock_builds=r.fock_builds,
                        phases_s={k: round(v, 4) for k, v in r.timings.items()}, _g=g)
    base_e, base_g = res["fp64_eager"]["energy"], res["fp64_eager"]["_g"]
    for tag, v in res.items():
        v["abs_dE_vs_fp64_Eh"] = abs(v["energy"] - base_e)
        v["max_abs_dgrad_vs_fp64"] = float(np.abs(v.pop("_g") - base_g).max())
    best = min(res, key=lambda k: res[k]["seconds_per_molecule"])
    # Kohn-Sham energy + gradient of a C40H82 chain in 6-31G** (1010 basis
    # functions), B3LYP, on QUICK's SG1 grid and on the 75 x 302 Becke grid;
    # the gradient includes the XC term (grid moving with the atoms)
    from quick_b200.molecule import linear_alkane
    alk = linear_alkane(40, seed=0)
    kohn_sham = {"workload": "C40H82 6-31G** (1010 basis functions), B3LYP, seeded torsions", "grids": {}}
    for grid, gname in ((1, "sg1"), (2, "becke_75x302")):
        ks = []
        for _ in range(2):
            barrier(ws)
            r, g = scf.run_rhf_device(alk, "6-31G**", 1e-10, 1e-20, conv=1e-7, device=local, method=1, gradient=True,
                                      session=sess, xc_grid=grid)
            ks.append((r, g))
        r, g = ks[-1]
        kohn_sham["grids"][gname] = {
            "seconds_per_molecule": max_over_ranks(r.seconds, ws), "energy": r.energy, "iterations": r.iterations,
            "converged": bool(r.converged), "phases_s": {k: round(v, 4) for k, v in r.timings.items()},
            "max_abs_gradient": float(np.abs(g).max()),
            "translational_sum": float(np.abs(g.reshape(-1, 3).sum(axis=0)).max())}
    kohn_sham["note"] = ("energy + gradient (one-electron, two-electron with 0.2 exchange, XC with basis-centre, "
                         "point and partition-weight terms); second of two runs per grid")
    # (H2O)32 in cc-pVTZ (2080 Cartesian functions, f shells on O): the RHF
    # energy all-FP64, and energy + gradient with the mixed split and delta-D
    tz = {}
    for tag, kw in (("fp64_energy", dict(gradient=False)),
                    ("mixed_delta_d", dict(gradient=True, mixed_cut=MIXED_CUT, incremental=True))):
        barrier(ws)
        r, g = scf.run_rhf_device(m, "cc-pVTZ", 1e-10, 1e-20, conv=1e-7, device=local, session=sess, **kw)
        tz[tag] = {"seconds_per_molecule": max_over_ranks(r.seconds, ws), "energy": r.energy,
                   "iterations": r.iterations, "converged": bool(r.converged),
                   "phases_s": {k: round(v, 3) for k, v in r.timings.items()}}
        if g is not None:
            tz[tag]["max_abs_gradient"] = float(np.abs(g).max())
            tz[tag]["translational_sum"] = float(np.abs(g.reshape(-1, 3).sum(axis=0)).max())
    tz["mixed_delta_d"]["abs_dE_vs_fp64_Eh"] = abs(tz["mixed_delta_d"]["energy"] - tz["fp64_energy"]["energy"])
    cc_pvtz = {"workload": "(H2O)32 cc-pVTZ (2080 basis functions), RHF, density RMS 1e-7",
               "variants": tz, "note": "SCF+grad s/mol with f shells (mixed_delta_d); all-FP64 energy for |dE|"}
    sess.close()
    return {"metric": "SCF+grad s/mol (RHF energy + analytic gradient)", "unit": "s/mol",
            "higher_is_better": False, "value": res[best]["seconds_per_molecule"], "best": best,
            "workload": "(H2O)32 6-31G** (800 basis functions), seeded 4x4x2 cluster",
            "molecules_timed_per_variant": nmol,
            "mixed_vs_fp64_speedup": res["fp64"]["seconds_per_molecule"] / res["mixed"]["seconds_per_molecule"],
            "mixed_delta_d_vs_fp64_speedup": res["fp64"]["seconds_per_molecule"]
            / res["mixed_delta_d"]["seconds_per_molecule"],
            "variants": res,
            "kohn_sham": kohn_sham,
            "cc_pvtz": cc_pvtz,
            "note": "SAD guess (atomic densities cached per element), GPU one-electron integrals, GPU Fock builds "
                    "with the density screen on the device, one-electron + two-electron gradient on the GPU; "
                    "fp64_eager: DIIS + cuSOLVER diagonalisation per iteration with a host convergence test; the "
                    "other variants replay each iteration from a CUDA graph (device DIIS solve, SP2 "
                    "purification); wall clock, |dE| and |dg| against fp64_eager"}


def run_batch(args, ws, rank, local, nmol=None):
    """Molecules/s for many small closed-shell molecules: (H2O)_n clusters,
    n uniform in 1..12 (seeded), 6-31G*, RHF energy + analytic gradient each
    (density RMS 1e-8).  Two ways: one molecule after another through one open
    session (device SCF from the SAD guess, gradient), and all of them
    advanced together (scf.run_batch_rhf: one batched Fock build per
    iteration for the whole batch, batched DIIS and purification, one batched
    two-electron gradient), with the energies of the two compared.  Molecules
    are split across ranks with no collective (weak scaling: each rank takes
    its own list)."""
    import torch
    from quick_b200 import capi, scf
    from quick_b200.molecule import water_cluster_n
    torch.cuda.set_device(local)
    nmol = nmol or args.batch
    sizes = batch_sizes(nmol, rank)
    mols = [water_cluster_n(int(k), seed=1000 * rank + i) for i, k in enumerate(sizes)]
    sess = capi.Session(local)
    try:
        scf.run_rhf_device(mols[0], "6-31G*", 1e-10, 1e-20, conv=1e-8, device=local, session=sess)   # warm-up
        barrier(ws)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        iters, nconv, e_seq = 0, 0, []
        for mol in mols:
            r, g = scf.run_rhf_device(mol, "6-31G*", 1e-10, 1e-20, conv=1e-8, device=local, session=sess)
            iters += r.iterations
            nconv += int(r.converged)
            e_seq.append(r.energy)
        torch.cuda.synchronize()
        sec = max_over_ranks(time.perf_counter() - t0, ws)
        # all molecules together (a warm-up batch of eight first)
        scf.run_batch_rhf(mols[:8], "6-31G*", 1e-10, 1e-20, conv=1e-8, device=local, session=sess)
        barrier(ws)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        res, grads, tim = scf.run_batch_rhf(mols, "6-31G*", 1e-10, 1e-20, conv=1e-8, device=local, session=sess)
        torch.cuda.synchronize()
        sec_b = max_over_ranks(time.perf_counter() - t0, ws)
    finally:
        sess.close()
    e_b = np.array([r.energy for r in res])
    batched = {"value": nmol * ws / sec_b, "unit": "molecules/s", "seconds": sec_b,
               "phases_s": {k: round(v, 4) for k, v in tim.items()},
               "converged": int(sum(r.converged for r in res)),
               "mean_iterations": float(np.mean([r.iterations for r in res])),
               "max_abs_dE_vs_one_at_a_time_Eh": float(np.abs(e_b - np.array(e_seq)).max()),
               "speedup_vs_one_at_a_time": sec / sec_b,
               "note": "one batched Fock build (one screen launch + one launch per angular class) per SCF "
                       "iteration for all molecules, delta-D builds, batched DIIS + SP2 purification, one "
                       "batched two-electron gradient; wall clock including uploads and set-up"}
    return {"metric": "molecules/s (RHF energy + gradient, (H2O)_n n~U[1,12], 6-31G*)", "unit": "molecules/s",
            "value": nmol * ws / sec, "seconds": sec, "molecules_per_rank": nmol, "n_gpus": ws,
            "scaling": "weak", "converged": nconv, "mean_iterations": iters / nmol,
            "basis_functions": [int(19 * k) for k in (sizes.min(), sizes.max())],
            "note": "value: one molecule after another in one session; batched: all advanced together",
            "batched": batched}


def run_xc(args, ws, rank, local, sess=None):
    """B3LYP XC quadrature (gpu_getxc_'s work, qb_xc_device) on the workload
    molecule's SG1 grid: device time per call with the grid resident, L2
    flushed before every call; end to end through gpu_getxc_ with host
    buffers."""
    import torch
    from quick_b200 import capi
    from quick_b200.basis import build_basis, sigrad2
    from quick_b200.molecule import water_cluster

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    stream = torch.cuda.Stream(dev)
    torch.cuda.set_stream(stream)
    m = water_cluster(WORKLOAD["grid"], seed=WORKLOAD["seed"])
    b = build_basis(m.symbols, WORKLOAD["basis"])
    n = b.nbasis
    own = sess is None
    if own:
        sess = capi.Session(local)
    lib = capi.lib()
    lib.qb_set_stream(capi.C.c_void_p(stream.cuda_stream))
    sess.upload_molecule(m, b)
    sg = np.ascontiguousarray(sigrad2(b))
    # a positive semi-definite closed-shell density 2 C C^T (rho >= 0 everywhere)
    rng = np.random.default_rng(WORKLOAD["seed"])
    C = rng.standard_normal((n, m.n_electrons // 2)) * 0.05
    D = np.asfortranarray(2.0 * C @ C.T)
    O0 = np.zeros((n, n), order="F")
    sess.getxc(O0, D, sg, method=1)                  # builds the grid once
    grid_ms = sess.xc_stats()["ms_grid"]
    dD = torch.from_numpy(np.ascontiguousarray(D)).to(dev)
    dV = torch.zeros((n, n), dtype=torch.float64, device=dev)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
    exc, nal = capi.C.c_double(0), capi.C.c_double(0)

    def step():
        dV.zero_()
        rc = lib.qb_xc_device(capi.C.c_void_p(dD.data_ptr()), capi._ptr(sg), capi.C.c_void_p(dV.data_ptr()),
                              capi.C.byref(exc), capi.C.byref(nal))
        if rc:
            capi.check()

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    barrier(ws)
    l0 = lib.qb_launch_count()
    e0 = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    e1 = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    for i in range(args.steps):
        flush.zero_()
        e0[i].record(stream)
        step()
        e1[i].record(stream)
    torch.cuda.synchronize()
    barrier(ws)
    launches = lib.qb_launch_count() - l0
    ms = max_over_ranks(float(np.mean([a.elapsed_time(c) for a, c in zip(e0, e1)])), ws)
    st = sess.xc_stats()
    # end to end: gpu_upload_method_ + gpu_upload_calculated_ + gpu_getxc_ from pinned host memory
    pinD = torch.from_numpy(np.asfortranarray(D).ravel(order="F").copy()).pin_memory()
    pinO = torch.zeros(n * n, dtype=torch.float64).pin_memory()
    co = torch.zeros(1, dtype=torch.float64)
    ptr = lambda t: capi.C.c_void_p(t.data_ptr())  # noqa: E731
    one = capi.C.byref
    ee = capi.C.c_double(0)
    ec0, ec1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    barrier(ws)
    torch.cuda.synchronize()
    ec0.record(stream)
    for i in range(args.steps):
        lib.gpu_upload_method_(one(capi.C.c_int(1)))
        lib.gpu_upload_calculated_(ptr(pinO), ptr(co), ptr(co), ptr(pinD))
        ee.value = 0.0
        lib.gpu_getxc_(one(capi.C.c_int(1)), capi._ptr(sg), one(ee), one(capi.C.c_double(0)),
                       one(capi.C.c_double(0)), ptr(pinO))
    ec1.record(stream)
    torch.cuda.synchronize()
    capi.check()
    e2e_ms = max_over_ranks(ec0.elapsed_time(ec1) / args.steps, ws)
    hbm, hbm_src = measured_hbm_gbs()
    peak64 = capi.C.c_double(0)
    lib.qb_fma_peak(1, capi.C.byref(peak64))
    gbs = st["alg_bytes"] / (ms * 1e-3) / 1e9
    tfl = st["gemm_flops"] / (ms * 1e-3) / 1e12
    if own:
        sess.close()
    return {
        "metric": "XC quadrature grid points/s (SG1, B3LYP, FP64)",
        "value": st["npts"] * ws / (ms * 1e-3), "unit": "points/s", "ms_per_call": ms,
        "config": {"workload": "(H2O)32 6-31G** B3LYP XC quadrature, QUICK SG1 grid", "grid_points": st["npts"],
                   "chunks": st["nchunks"], "grid_build_ms": grid_ms, "l2": "flushed (256 MB write) before every call"},
        "e2e": {"value": st["npts"] * ws / (e2e_ms * 1e-3), "unit": "points/s", "ms_per_call": e2e_ms,
                "h2d_bytes_per_step": int(2 * n * n * 8 + n * 8), "d2h_bytes_per_step": int(n * n * 8)},
        # the three FP64 DGEMMs per chunk take over half the time (profiles/
        # xc_quadrature_water32_631gss.md), so the bound is the FP64 pipe:
        # achieved = the FLOPs those GEMMs execute per call / call time
        "roofline": {"bound": "fp64", "achieved": tfl, "peak": peak64.value / 1e3, "unit": "TFLOP/s",
                     "frac": tfl / (peak64.value / 1e3) if peak64.value else None, "traffic": None,
                     "peak_source": "measured: FP64 FMA-chain probe run in this process (qb_fma_peak)",
                     "gemm_flops_per_call": st["gemm_flops"], "alg_flops_per_call": st["alg_flops"],
                     "hbm_gbs_of_alg_bytes": gbs, "hbm_peak_gbs": hbm, "hbm_peak_source": hbm_src,
                     "alg_bytes_per_call": st["alg_bytes"]},
        "gpu_launches": int(launches),
        "exc": exc.value,
    }


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--classes", action="store_true", help="add per-class quartet counts")
    ap.add_argument("--batch", type=int, default=256, help="molecules in the batch line")
    ap.add_argument("--part", default="all", choices=["all", "fock", "xc", "scf", "batch", "quick-gpu"],
                    help="fock: the Fock build line only; xc: the XC quadrature line only; "
                         "scf: the SCF+gradient line only; batch: the many-small-molecules line only; "
                         "quick-gpu (with --impl reference): QUICK's own GPU path on the Fock-build workload")
    ap.add_argument("--no-quick-gpu", action="store_true", help="skip the reference_gpu object")
    ap.add_argument("--grid", default=None,
                    help="water-cluster grid of the workload, e.g. 2,2,2 for (H2O)8 (default 4,4,2: (H2O)32); "
                         "smaller cases are for profiling only")
    ap.add_argument("--basis", default=None,
                    help="basis set of the workload (default 6-31G**); others, e.g. cc-pVTZ, are for profiling only")
    args = ap.parse_args()
    if args.grid or args.basis:
        g = tuple(int(x) for x in args.grid.split(",")) if args.grid else WORKLOAD["grid"]
        WORKLOAD["grid"] = g
        WORKLOAD["basis"] = args.basis or WORKLOAD["basis"]
        WORKLOAD["name"] = "(H2O)%d %s RHF Fock build" % (g[0] * g[1] * g[2], WORKLOAD["basis"])
    threads = os.cpu_count() or 1
    if args.impl == "reference" and args.part == "quick-gpu":
        # QUICK's own GPU path only (run by the default line in a process of its own)
        print(json.dumps(gpu_reference(args.steps, args.warmup, int(os.environ.get("LOCAL_RANK", "0")))))
        return
    if args.impl == "reference":
        # QUICK's own kernel on the host cores; under torchrun rank 0 alone
        # runs it and the other ranks exit without work (no process group)
        ws = int(os.environ.get("WORLD_SIZE", "1"))
        if int(os.environ.get("RANK", "0")) == 0:
            qps, nq, sec, raw = cpu_reference(threads, steps=args.steps, warmup=args.warmup)
            sample = ("%d full Fock builds of %s (%d unique shell quartets, %d iclass calls, per build); "
                      "QUICK's gpu_get2e_subs.h kernel and gpu.cu bridge compiled for the host cores; warm-up "
                      "builds on %s" % (args.steps, WORKLOAD["name"], nq, raw, WARMUP_SAMPLE["name"]))
            out = {"impl": "reference", "metric": "Fock-build shell quartets/s (FP64)", "value": qps,
                   "unit": "quartets/s", "n_gpus": ws, "steps": args.steps, "warmup": args.warmup,
                   "ms_per_step": sec * 1e3, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                   "dtype": "f64", "data": "synthetic: seeded (H2O)32 geometry, model density",
                   "config": workload_config(800, nq),
                   "cpu_baseline": {"value": qps, "unit": "quartets/s", "cores": threads, "kind": "reference",
                                    "sample": sample},
                   "e2e": {"value": qps, "unit": "quartets/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
            import torch
            if torch.cuda.is_available() and not args.no_quick_gpu:
                # QUICK's own CUDA path on the same box's GPU, beside its host-core run
                out["reference_gpu"] = quick_gpu_subprocess(3, 1, int(os.environ.get("LOCAL_RANK", "0")))
            print(json.dumps(out))
        return
    ws, rank, local = dist_setup()
    if args.part in ("xc", "scf", "batch"):
        out = {"xc": run_xc, "scf": run_scf, "batch": run_batch}[args.part](args, ws, rank, local)
        if rank == 0:
            print(json.dumps(out))
        if ws > 1:
            import torch.distributed as dist
            dist.destroy_process_group()
        return
    out = run_ours(args, ws, rank, local)
    if args.part == "all":
        out["xc"] = run_xc(args, ws, rank, local)
        out["scf"] = run_scf(args, ws, rank, local)
        out["batch"] = run_batch(args, ws, rank, local)
    if rank == 0 and not args.no_cpu_baseline:
        qps, nq, sec, raw = cpu_reference(threads)
        out["cpu_baseline"] = {"value": qps, "unit": "quartets/s", "cores": threads, "kind": "reference",
                               "sample": "one full Fock build of %s (%d unique shell quartets, %.2f s); QUICK's "
                                         "gpu_get2e_subs.h kernel and gpu.cu bridge compiled for the host cores"
                                         % (WORKLOAD["name"], nq, sec),
                               "quartets_equal_gpu_count": nq == out["config"]["quartets_per_step"]}
    if rank == 0 and ws == 1 and not args.no_quick_gpu:
        out["reference_gpu"] = quick_gpu_subprocess(3, 1, local)
        if "value" in out["reference_gpu"]:
            rg = out["reference_gpu"]
            rg["e2e_speedup_of_this_build"] = out["e2e"]["value"] / rg["value"]
            rg["kernel_speedup_of_this_build"] = out["value"] / rg["kernel_quartets_per_s"]
            gr = out.get("gradient", {})
            if "e2e_ms_per_call" in gr:
                rg["gradient"]["e2e_speedup_of_this_build"] = rg["gradient"]["ms_per_call"] / gr["e2e_ms_per_call"]
                rg["gradient"]["kernel_speedup_of_this_build"] = rg["gradient"]["kernel_ms"] / gr["kernel_ms"]
            if "xc" in out and "e2e" in out["xc"]:
                rg["xc"]["e2e_speedup_of_this_build"] = rg["xc"]["ms_per_call"] / out["xc"]["e2e"]["ms_per_call"]
                rg["xc"]["abs_dExc_vs_this_build"] = abs(rg["xc"]["exc"] - out["xc"]["exc"])
    if rank == 0:
        print(json.dumps(out))
    if ws > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


def quick_gpu_subprocess(steps, warmup, device):
    """gpu_reference in a process of its own (QUICK's library never shares
    a process with this package's): its JSON object, or the reason it is
    missing."""
    if not os.path.exists(os.path.join(ROOT, "oracle", "_ref", "gpu", "libquickref.so")):
        return {"unavailable": "QUICK's GPU build (oracle/_ref/gpu) was not built"}
    env = dict(os.environ, LOCAL_RANK=str(device))
    for k in ("RANK", "WORLD_SIZE", "MASTER_ADDR", "MASTER_PORT"):
        env.pop(k, None)
    p = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--part",
                        "quick-gpu", "--steps", str(steps), "--warmup", str(warmup)],
                       capture_output=True, text=True, env=env, timeout=900)
    for line in reversed(p.stdout.splitlines()):
        if line.startswith("{"):
            return json.loads(line)
    return {"unavailable": "QUICK's GPU path exited %d: %s" % (p.returncode, (p.stderr or p.stdout)[-300:])}


if __name__ == "__main__":
    main()
