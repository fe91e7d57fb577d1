"""Benchmark: k-point H+O setups per second on the 8-atom Si cell.

Workload (one "step"): the first-variational H and O of all 27 k-points of
the shifted 3x3x3 mesh of the 8-atom simple-cubic Si cell (a = 10.26 Bohr,
U(+-0.02) Bohr displacements, rgkmax 8, lmaxapw = lmaxmat = 10, APW order 2,
3 lo per l <= 2; N_G+k 968..1016, nmat 1184..1232), seeded synthetic SCF
inputs.  One setup = match + MT APW-APW/APW-lo/lo-lo + interstitial + the full
Hermitian H and O, as seceqnfv.f90:76-77 leaves them.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

``value``: setups/s with every input resident in HBM (the device-pointer
entry point), max over ranks; ``e2e``: the same through the host-pointer
entry point, the H2D of igpig/vgpc and the D2H of H and O inside the timed
region.  Multi-GPU: one process per GPU, each rank sets up its own 27 k-points
(weak scaling, no collective on the data path).
``--impl reference`` times the CPU restatement of the reference's algorithm
(the Fortran reference cannot be compiled here) on the host cores.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "k-pt H+O setups/s"
WORKLOAD = "si_cube8 8-atom Si, 27 k (3x3x3 shifted), rgkmax 8, lmaxapw 10, 3 lo/l<=2"


def _dist():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    return ws, rank


def _clock_sampler(stop, rows):
    cmd = ["nvidia-smi", "--query-gpu=index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
           "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
           "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap",
           "--format=csv,noheader,nounits", "-lms", "200"]
    try:
        p = subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
    except OSError:
        return
    try:
        while not stop.is_set():
            line = p.stdout.readline()
            if not line:
                break
            rows.append(line.strip())
    finally:
        p.terminate()
        try:
            p.wait(timeout=2)
        except Exception:
            p.kill()


def _clock_summary(rows, dev):
    sm, mx, reasons = [], None, set()
    for r in rows:
        f = [x.strip() for x in r.split(",")]
        if len(f) < 9 or f[0] != str(dev):
            continue
        try:
            sm.append(float(f[1]))
            mx = float(f[2])
        except ValueError:
            continue
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for n, v in zip(names, f[5:9]):
            if v.lower() == "active":
                reasons.add(n)
    if not sm:
        return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
    return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


def _measured_fp64_peak(torch):
    """cuBLAS DGEMM 8192^3 rate (TFLOP/s): the FP64 roofline denominator."""
    a = torch.randn(8192, 8192, dtype=torch.float64, device="cuda")
    b = torch.randn_like(a)
    for _ in range(2):
        a @ b
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    best = 0.0
    for _ in range(3):
        e0.record()
        a @ b
        e1.record()
        torch.cuda.synchronize()
        best = max(best, 2 * 8192 ** 3 / (e0.elapsed_time(e1) * 1e-3) / 1e12)
    del a, b
    torch.cuda.empty_cache()
    return best


def _measured_int8_peak(torch):
    """cuBLASLt int8 GEMM 8192^3 rate (TOP/s, torch._int_mm): the int8 tensor roofline denominator."""
    a = torch.randint(-127, 127, (8192, 8192), dtype=torch.int8, device="cuda")
    b = torch.randint(-127, 127, (8192, 8192), dtype=torch.int8, device="cuda")
    for _ in range(2):
        torch._int_mm(a, b)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    best = 0.0
    for _ in range(3):
        e0.record()
        torch._int_mm(a, b)
        e1.record()
        torch.cuda.synchronize()
        best = max(best, 2 * 8192 ** 3 / (e0.elapsed_time(e1) * 1e-3) / 1e12)
    del a, b
    torch.cuda.empty_cache()
    return best


def _measured_int8_sustained(torch, seconds=4.0):
    """cuBLASLt int8 GEMM 8192^3 back to back for `seconds` (TOP/s, with the
    clocks seen): the denominator for a kernel that runs for seconds under
    the power cap, as the 216-atom H/O kernel does."""
    a = torch.randint(-127, 127, (8192, 8192), dtype=torch.int8, device="cuda")
    b = torch.randint(-127, 127, (8192, 8192), dtype=torch.int8, device="cuda")
    torch._int_mm(a, b)
    torch.cuda.synchronize()
    rows, stop = [], threading.Event()
    th = threading.Thread(target=_clock_sampler, args=(stop, rows), daemon=True)
    th.start()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    n = 0
    t0 = time.perf_counter()
    e0.record()
    while time.perf_counter() - t0 < seconds:
        for _ in range(8):
            torch._int_mm(a, b)
        n += 8
        torch.cuda.synchronize()
    e1.record()
    torch.cuda.synchronize()
    stop.set()
    th.join(timeout=3)
    v = n * 2 * 8192 ** 3 / (e0.elapsed_time(e1) * 1e-3) / 1e12
    del a, b
    torch.cuda.empty_cache()
    return v, _clock_summary(rows, torch.cuda.current_device())


def _int8_from_bf16_peaks(achieved):
    """The int8 dense rate as twice MEASURED_PEAKS.json's bf16 GEMM figures
    (that file has no int8 entry; the tensor cores' int8 rate is twice the
    bf16 rate), beside the in-run cuBLASLt int8 peaks."""
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            mp = json.load(f)
        b, bs = 2.0 * float(mp["bf16_tflops"]), 2.0 * float(mp["bf16_tflops_sustained"])
    except (OSError, KeyError, ValueError):
        return {}
    return {"peak_2x_bf16_measured_peaks": b, "frac_of_2x_bf16": achieved / b,
            "peak_2x_bf16_sustained_measured_peaks": bs, "frac_of_2x_bf16_sustained": achieved / bs}


def _hbm_peak():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"])
    except (OSError, KeyError, ValueError):
        return 6650.0      # earlier measurement on this pool's B200s


def split_scheme(args, sys_):
    """(int8 planes per operand, int8 products per output tile, dtype text,
    precision text) of the split-precision mode args.precision."""
    if args.precision == "ozaki":
        S = args.slices
        return (S, S * (S + 1) // 2, "i8 slices, f64 recombination",
                "split int8 x%d slices (tcgen05), FP64 recombination" % S)
    from exciting_b200.fvsystem import ozaki_moduli
    K = sum(sys_.basis.napw_atom(a) for a in range(sys_.natmtot))
    ps, _, b, bx, h = ozaki_moduli(args.moduli, K, sys_.basis.maxaa)
    n = len(ps)
    return (n, n, "i8 residues mod %d coprime moduli, CRT in 64-bit fixed point, f64 scaling" % n,
            "split int8, residues modulo %d moduli (columns scaled by their 2-norms to %d bits, %d headroom bits "
            "in the 64-bit recombination; tcgen05), Chinese-remainder recombination" % (n, b, h))


def ozaki_tiles128(g, cols=64):
    """128-row upper residue tiles of one k-point (128 x cols)."""
    n = g.ngp
    return sum(1 for ib in range((n + 127) // 128) for jb in range((n + cols - 1) // cols)
               if jb * cols + cols - 1 >= ib * 128)


def residue_bytes(sys_, g, moduli):
    """Algorithmic DRAM bytes of the residue kernel for one k-point: the
    residues of Ar, Ai, Br, Bi (npad rows x kp8 bytes per modulus) read once
    and the residues of the four H/O values written once (128 x 64 bytes per
    value, tile and modulus)."""
    K = sum(sys_.basis.napw_atom(a) for a in range(sys_.natmtot))
    kp8 = (K + 255) // 256 * 256
    npad = (g.ngp + 63) // 64 * 64
    return 4.0 * moduli * npad * kp8 + 4.0 * moduli * 128 * 64 * ozaki_tiles128(g)


def ozaki_int8_ops(sys_, gks, products, cols=32):
    """int8 MMA operations the split-precision H/O kernel issues: per 128 x
    cols tile (B operand [Br|Bi|Ar|Ai] -> N = 4 cols), `products` int8
    products (S(S+1)/2 slice pairs, or one per modulus) x two A operands
    (Ar, Ai) x 2 x 128 x N x kp8 (K padded to 256)."""
    K = sum(sys_.basis.napw_atom(a) for a in range(sys_.natmtot))
    kp8 = (K + 255) // 256 * 256
    tiles = 0
    for g in gks:
        n = g.ngp
        for ib in range((n + 127) // 128):
            for jb in range((n + cols - 1) // cols):
                if jb * cols + cols - 1 >= ib * 128:
                    tiles += 1
    return tiles * products * 2.0 * 2 * 128 * (4 * cols) * kp8


HO_KERNEL = {"ozaki_mod": "oz_res_kernel (residue tiles, tcgen05.mma kind::i8) + oz_crt_kernel (96-bit CRT), "
                          "MT contraction phase",
             "ozaki": "oz_mma_kernel (tcgen05.mma kind::i8, FP64 fold), MT contraction phase"}


def ho_kernel(precision, kernel_config):
    if precision == "ozaki_mod" and kernel_config >= 0 and (kernel_config & 8):
        how = "persistent paced clusters, " if kernel_config & 2 else ""
        return HO_KERNEL[precision].replace("oz_res_kernel (residue tiles", "oz_res2_kernel (256 x 64 residue tiles "
                                            "on SM pairs, %stcgen05.mma.cta_group::2" % how)
    return HO_KERNEL[precision]


def ho_tile_cols(precision, kernel_config):
    """Columns of the H/O tiles: 64 or 32 for the modular residue tiles
    (configuration bit 0; the two-SM tiles of bit 3 are 64 wide), 32 for the
    slice kernel.  The operation count is that of the 128-row tiles either
    way: the two-SM tiles' extra tiles below the diagonal are not counted."""
    if precision == "ozaki_mod":
        return 32 if (kernel_config & 1) and not (kernel_config & 8) else 64
    return 32


# DRAM bytes of the dominant kernel, from ncu captures (dram__bytes_read.sum +
# dram__bytes_write.sum) of the same kernels; a kernel change needs a new
# capture.  The 8-atom batch, per k-point (a 2 k-point capture divided by 2;
# the traffic grows with the k-points: each k-point's operands are read once
# and its H/O written once):
#   slices, oz_mma_kernel<OZ_HO,2,2>, 7 slices: 131.6 MB read + 35.2 MB written;
#   moduli, oz_res_kernel<64> (configurations without bit 3): 218.4 MB read +
#     47.4 MB written; oz_res2_kernel<64> (bit 3): 253.9 MB + 56.9 MB;
#   FP64, zgemm_dmma_kernel<1> + <2>, 6 k-points: 673.5 MB read + 143.1 MB written.
# The 216-atom cell, per k-point (one launch, captured at full size in one
# pass): oz_res2_kernel<64> in configuration 10 (paced persistent pairs),
# 1.23 TB read + 19.6 GB written; configuration 8, 4.61 TB + 19.9 GB.
PROFILED_DRAM_BYTES_PER_K = {"ozaki": (131.6e6 + 35.2e6) / 2, "fp64": (673.5e6 + 143.1e6) / 6,
                             "ozaki_mod": (218.4e6 + 47.4e6) / 2, "ozaki_mod_pairs": (253.9e6 + 56.9e6) / 2}
PROFILED_DRAM_BYTES_216 = {10: 1.23e12 + 19.6e9, 8: 4.61e12 + 19.9e9}


def profiled_traffic_per_k(precision, kernel_config):
    if precision == "ozaki_mod" and kernel_config >= 0 and (kernel_config & 8):
        return PROFILED_DRAM_BYTES_PER_K["ozaki_mod_pairs"]
    return PROFILED_DRAM_BYTES_PER_K[precision]


def main_bytes(sys_, gks, precision, slices):
    """Algorithmic DRAM bytes of the MT contraction launch(es): operands read
    once (int8 slices or residues of Ar, Ai, Br, Bi, `slices` planes each; or
    the FP64 A and B planes) and the N x N block of H and O written once."""
    K = sum(sys_.basis.napw_atom(a) for a in range(sys_.natmtot))
    total = 0.0
    for g in gks:
        n = g.ngp
        npad = (n + 63) // 64 * 64
        if precision != "fp64":
            kp8 = (K + 255) // 256 * 256
            total += 4.0 * slices * npad * kp8
        else:
            total += 4.0 * 8 * K * npad
        total += 2.0 * 16 * n * n
    return total


def main_flops(sys_, gks):
    """Algorithmic flops of the MT contraction stage (upper triangles of A^H B and A^H A):
    sum over k of 8 N (N+1) K, K = sum_a m_a."""
    K = sum(sys_.basis.napw_atom(a) for a in range(sys_.natmtot))
    return sum(8.0 * g.ngp * (g.ngp + 1) * K for g in gks)


def setup_flops(sys_, gks):
    """All MT flops of a setup (the unit-of-work figure): h_a A_a + both upper
    triangles + APW-lo rows."""
    b = sys_.basis
    tot = 0.0
    for g in gks:
        n = g.ngp
        for a in range(sys_.natmtot):
            m = b.napw_atom(a)
            lo = b.losize[b.atom_species[a]]
            tot += 8.0 * m * m * n + 8.0 * n * (n + 1) * m + 8.0 * lo * m * n
    return tot


def cpu_sample(sys_, gks, budget_s=12.0):
    """Time the oracle (CPU restatement) on a bounded sample of the workload."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import lapw_oracle as O
    O.lib()
    O.hamiltonandoverlapsetup(sys_, gks[0])       # warm-up
    n = 0
    t0 = time.perf_counter()
    while n < len(gks):
        O.hamiltonandoverlapsetup(sys_, gks[n])
        n += 1
        if time.perf_counter() - t0 > budget_s:
            break
    dt = time.perf_counter() - t0
    return n / dt, n, dt


def run_reference(args):
    """The CPU arm: the FP64 restatement of the path (the Fortran reference
    has no compiler on either machine) on the host cores, on the same
    workload, metric and unit as the GPU arm; each step a bounded sample of
    one k-point, extrapolated to the whole k-point.  Rank 0 only."""
    ws, rank = _dist()
    if rank != 0:
        return 0
    from exciting_b200 import workloads as W
    cores = os.cpu_count()
    if args.workload == "cube216":
        s = W.si_cube216()
        gks = s.gksets()
        for i in range(args.warmup):
            cpu_sample_216(s, gks[i % len(gks)], 1, 1000)
        vals = []
        for i in range(args.steps):
            full, _ = cpu_sample_216(s, gks[i % len(gks)], 1, 1000)
            vals.append(1.0 / full)
        value = float(np.median(vals))
        config = {"workload": WORKLOAD_216, "k_per_step": 1,
                  "kpoints": "Gamma, (1/2,0,0), (1/2,1/2,0), (1/2,1/2,1/2) in turn, one per step"}
        sample = ("per step one k-point in turn: match and the H and O zgemm pairs of 1 of 216 atoms plus "
                  "hmlistln/olpistln over 1000 G+k by the FP64 CPU restatement (C + OpenBLAS zgemm), "
                  "extrapolated linearly in atoms and by N(N+1) in G+k; the value is the median over steps; "
                  "the Fortran reference has no compiler here")
        ms = 1e3 / value
    else:
        s = W.si_cube8()
        gks = s.gksets()
        for _ in range(args.warmup):
            cpu_sample(s, gks, budget_s=1.0)
        vals = []
        for _ in range(args.steps):
            v, n, dt = cpu_sample(s, gks, budget_s=6.0)
            vals.append(v)
        value = float(np.median(vals))
        config = {"workload": WORKLOAD, "k_per_step": 27}
        sample = ("k-points of the 27-k set set up by the FP64 CPU restatement (C + OpenMP + OpenBLAS zgemm) "
                  "until 6 s elapse, per step; the Fortran reference has no compiler here")
        ms = 27.0 / value * 1e3
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "setups/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
        "higher_is_better": True, "scaling": "strong" if args.workload == "cube216" else "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic", "config": config,
        "cpu_baseline": {"value": value, "unit": "setups/s", "cores": cores, "kind": "port", "sample": sample},
        "e2e": {"value": value, "unit": "setups/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def launches_per_setup(precision):
    """Kernel launches of one batched setup call: match, (modular: the A column
    norms), the A split, the per-atom products, (modular: the B column norms),
    the B split, the H/O tiles (modular: residue tiles, then their
    recombination), the O APW-lo block and the lo-lo blocks; the FP64 path:
    match, four grouped DMMA products, APW-lo and lo-lo."""
    return 10 if precision == "ozaki_mod" else 7


def _e2e(args, st, stream, ig, vg, ngp, nmat, ws, barrier, mode="auto", pinned=True):
    """Setups/s through exs_setup_batched: pinned host igpig/vgpc in, host H/O out
    (pinned or pageable), H/O brought back in the given copy mode."""
    import ctypes

    import torch
    import torch.distributed as dist
    nk = len(ngp)
    st.set_host_copy_mode(mode)
    h_ig = torch.from_numpy(np.ascontiguousarray(ig)).pin_memory()      # (nk, ngkmax) == Fortran (ngkmax, nk)
    h_vg = torch.from_numpy(np.ascontiguousarray(vg)).pin_memory()      # (nk, ngkmax, 3) == Fortran (3, ngkmax, nk)
    if pinned:
        h_out = [(torch.empty(2 * m * m, dtype=torch.float64).pin_memory(),
                  torch.empty(2 * m * m, dtype=torch.float64).pin_memory()) for m in nmat]
    else:
        h_out = [(torch.empty(2 * m * m, dtype=torch.float64), torch.empty(2 * m * m, dtype=torch.float64))
                 for m in nmat]
    ngp_np = np.array(ngp, dtype=np.int32)
    hpp = (ctypes.c_void_p * nk)(*[a.data_ptr() for a, _ in h_out])
    opp = (ctypes.c_void_p * nk)(*[b.data_ptr() for _, b in h_out])

    def step_host():
        rc = st.lib.exs_setup_batched(st.ctx, nk, ngp_np.ctypes.data_as(ctypes.c_void_p),
                                      ctypes.c_void_p(h_ig.data_ptr()), ctypes.c_void_p(h_vg.data_ptr()), hpp, opp)
        if rc < 0:
            raise RuntimeError(st.lib.exs_last_error(st.ctx))

    for _ in range(max(1, args.warmup)):
        step_host()
    torch.cuda.synchronize()
    barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with torch.cuda.stream(stream):
        e0.record(stream)
        for _ in range(args.steps):
            step_host()
        e1.record(stream)
    torch.cuda.synchronize()
    t = torch.tensor([e0.elapsed_time(e1)], dtype=torch.float64, device="cuda")
    if ws > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    value = ws * nk * args.steps / (float(t.item()) * 1e-3)
    h2d = ig.nbytes + vg.nbytes
    packed = mode == "packed" or (mode == "auto" and not pinned)

    def upper_bytes(m):   # rows 0 .. j0+63 of each block of 64 columns
        return sum(16 * min(m, j0 + 64) * (min(m, j0 + 64) - j0) for j0 in range(0, m, 64))

    d2h = sum(2 * (upper_bytes(m) if mode == "upper" else 16 * (m * (m + 1) // 2 if packed else m * m))
              for m in nmat)
    st.set_host_copy_mode("auto")
    return value, h2d, d2h


def hmlint_flops(sys_, rad):
    """FP64 flops of the radial integrals of hmlint: per atom, lmmaxvr
    potential channels x nrad^2 function pairs x nrmt points x 2 (one FMA),
    plus the kinetic channel (two FMAs per point)."""
    b, cr = sys_.basis, sys_.crystal
    fl = 0.0
    for ias in range(cr.natmtot):
        is_ = cr.atom_species[ias]
        nrad = sum(b.apword[is_][l] for l in range(b.lmaxmat + 1)) + len(b.lorbl[is_])
        fl += (rad.lmmaxvr * 2.0 + 4.0) * nrad * nrad * float(rad.nrmt[is_])
    return fl


def hmlint_leg(args, st, sys_, stream, torch):
    """exs_hmlint_device timed with CUDA events on the context's stream,
    exs_hmlint (host arrays in, integrals out) by wall clock, and on cube8 the
    oracle's CPU restatement of hmlint beside them.  Restores the synthetic
    integrals of the setup afterwards."""
    from exciting_b200 import workloads as W
    rad = W.mt_radial(sys_)
    dev = {k: torch.from_numpy(np.asfortranarray(getattr(rad, k)).ravel(order="F")).cuda()
           for k in ("apwfr", "lofr", "veffmt")}
    torch.cuda.synchronize()

    def call():
        st.hmlint_device(rad, dev["apwfr"].data_ptr(), dev["lofr"].data_ptr(), dev["veffmt"].data_ptr())

    for _ in range(max(3, args.warmup)):
        call()
    st.synchronize()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    n = 20
    with torch.cuda.stream(stream):
        e0.record(stream)
        for _ in range(n):
            call()
        e1.record(stream)
    st.synchronize()
    torch.cuda.synchronize()
    dev_ms = e0.elapsed_time(e1) / n
    st.hmlint(rad)
    t0 = time.perf_counter()
    nrep = 5
    for _ in range(nrep):
        st.hmlint(rad)
    e2e_ms = (time.perf_counter() - t0) * 1e3 / nrep
    cpu = None
    if not args.skip_cpu and sys_.natmtot <= 8:
        sys.path.insert(0, os.path.join(os.path.dirname(os.path.abspath(__file__)), "oracle"))
        import lapw_oracle as O
        t0 = time.perf_counter()
        O.hmlint(sys_, rad)
        dt = time.perf_counter() - t0
        cpu = {"value": sys_.natmtot / dt, "unit": "atoms/s", "cores": 1, "kind": "port",
               "sample": f"all {sys_.natmtot} atoms in {dt:.2f} s by the oracle's C restatement of "
                         "mt_kin + mt_pot (one fderiv spline per radial product, as the reference)"}
    st.set_scf_inputs()
    fl = hmlint_flops(sys_, rad)
    peak64 = _measured_fp64_peak(torch)
    nin = sum(getattr(rad, k).size for k in ("apwfr", "lofr", "veffmt")) * 8
    return {
        "kernels": "mt_radial_kernel + mt_angular_kernel (exs_hmlint_device)",
        "value": sys_.natmtot / (dev_ms * 1e-3), "unit": "atoms/s", "ms": dev_ms,
        "e2e": {"value": sys_.natmtot / (e2e_ms * 1e-3), "unit": "atoms/s", "ms": e2e_ms,
                "h2d_bytes": int(nin), "note": "exs_hmlint: pageable host inputs, integrals copied back"},
        "lmaxvr": rad.lmaxvr, "nrmt": int(rad.nrmt[0]),
        "roofline": {"bound": "fp64", "achieved": fl / (dev_ms * 1e-3) / 1e12, "peak": peak64,
                     "unit": "TFLOP/s", "frac": fl / (dev_ms * 1e-3) / 1e12 / peak64,
                     "flops": fl, "peak_source": "cuBLAS DGEMM 8192^3 measured in this run"},
        "cpu_baseline": cpu,
    }


def rttddft_leg(args, st, stream, torch, ngp, nmat, d_ig, d_vg, hp, op, step_device, sys_=None, gks=None):
    """exs_rttddft_updateham_device over the bench's k-points (setup + the
    field/momentum combination, momentum matrices resident) against the plain
    batched setup, both timed with CUDA events on the context's stream; the
    difference is the combination kernel, reported against measured HBM
    bandwidth (5 complex reads and 1 write per element)."""
    d_p = [torch.randn(6 * m * m, dtype=torch.float64, device="cuda") for m in nmat]
    pp = [t.data_ptr() for t in d_p]
    atot = np.array([0.3, -0.2, 0.5])

    def step():
        st.rttddft_updateham_device(ngp, d_ig.data_ptr(), d_vg.data_ptr(), atot, True, pp, hp, op)

    def timed(fn):
        for _ in range(max(3, args.warmup)):
            fn()
        st.synchronize()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        with torch.cuda.stream(stream):
            e0.record(stream)
            for _ in range(args.steps):
                fn()
            e1.record(stream)
        st.synchronize()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / args.steps

    t_rt = timed(step)
    comb_ms = float(st.last_timings()[5])     # CUDA events around the combination of the last step
    t_setup = timed(step_device)
    nbytes = 96.0 * sum(m * m for m in nmat)
    del d_p
    cpu = None
    if not args.skip_cpu and gks is not None:
        # the oracle's UpdateHam on a bounded sample: two k-points of the batch
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import lapw_oracle as O
        rng = np.random.default_rng(0)
        t0 = time.perf_counter()
        for g in gks[:2]:
            m = g.ngp + st.nlotot
            O.rttddft_updateham(sys_, g, atot, rng.standard_normal((m, m, 3)) + 0j)
        dt = time.perf_counter() - t0
        cpu = {"value": 2 / dt, "unit": "k-points/s", "cores": os.cpu_count(), "kind": "port",
               "sample": f"2 k-points in {dt:.2f} s by the oracle (setup restatement + the combination)"}
    # momentum matrices generated on the device (once per propagation), 9 k-points
    gen = None
    if gks is not None:
        from exciting_b200 import workloads as W
        rad = W.mt_radial(sys_)
        sub = gks[:9]
        al = [st.match(g)[0] for g in sub]
        st.rttddft_genpmat(sub, al, rad, outputs=False)          # warm-up (cuBLAS handle, buffers)
        t0 = time.perf_counter()
        st.rttddft_genpmat(sub, al, rad, outputs=False)
        dt = time.perf_counter() - t0
        gen = {"value": len(sub) / dt, "unit": "k-points/s", "ms": dt * 1e3, "k_points": len(sub),
               "note": "exs_rttddft_genpmat (pmatrad + genpmatbasisik), host matching coefficients in, "
                       "wall clock of the synchronous call"}
    return {"value": len(nmat) / (t_rt * 1e-3), "unit": "k-points/s", "ms_per_step": t_rt, "cpu_baseline": cpu,
            "genpmat": gen,
            "setup_ms_per_step": t_setup,
            "combine": {"kernel": "rt_combine_kernel", "ms_per_step": comb_ms, "bytes_per_step": nbytes,
                        "achieved": nbytes / (comb_ms * 1e-3) / 1e9, "unit": "GB/s", "peak": _hbm_peak(),
                        "frac": nbytes / (comb_ms * 1e-3) / 1e9 / _hbm_peak(),
                        "note": "CUDA events around the combination kernel of the last timed step"},
            "note": "exs_rttddft_updateham_device: UpdateHam's k-loop, calculate_overlap = .true."}


def run_ours(args, emit=True):
    """The 8-atom batch (27 k-points per step); with emit=False the JSON
    object is returned instead of printed (the secondary leg of the
    216-atom run, one process)."""
    import torch
    import torch.distributed as dist
    from exciting_b200 import workloads as W
    from exciting_b200.fvsystem import Setup

    ws, rank = _dist()
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if ws > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=120), device_id=torch.device("cuda", local))

    def barrier():
        if ws > 1:
            dist.barrier()

    s = W.si_cube8()
    gks = s.gksets()[: args.nk]
    nk = len(gks)
    st = Setup(s, max_batch=nk)
    if args.precision != "fp64":
        st.set_precision(args.precision, args.slices if args.precision == "ozaki" else args.moduli)
        planes, products, dtype_text, prec_text = split_scheme(args, s)
    stream = torch.cuda.Stream()
    st.set_stream(stream.cuda_stream)
    ngkmax, nlotot = st.ngkmax, st.nlotot
    ig = np.zeros((nk, ngkmax), dtype=np.int32)
    vg = np.zeros((nk, ngkmax, 3))
    for k, g in enumerate(gks):
        ig[k, : g.ngp] = g.igpig
        vg[k, : g.ngp] = g.vgpc.T
    d_ig = torch.from_numpy(ig).cuda()
    d_vg = torch.from_numpy(vg).cuda()
    ngp = [g.ngp for g in gks]
    nmat = [n + nlotot for n in ngp]
    d_h = [torch.empty(2 * m * m, dtype=torch.float64, device="cuda") for m in nmat]
    d_o = [torch.empty(2 * m * m, dtype=torch.float64, device="cuda") for m in nmat]
    hp = [t.data_ptr() for t in d_h]
    op = [t.data_ptr() for t in d_o]

    def step_device():
        st.setup_batched_device(ngp, d_ig.data_ptr(), d_vg.data_ptr(), hp, op)

    # ---- kernel configuration chosen by the library's autotuner on this batch (or given)
    if args.kernel_config >= 0 and args.precision != "fp64":
        st.set_kernel_config(args.kernel_config)
        tuned = args.kernel_config
    else:
        tuned = st.autotune(ngp, d_ig.data_ptr(), d_vg.data_ptr(), hp, op)

    # ---- device-resident timing
    for _ in range(args.warmup):
        step_device()
    st.synchronize()
    rows, stop = [], threading.Event()
    th = threading.Thread(target=_clock_sampler, args=(stop, rows), daemon=True)
    th.start()
    time.sleep(0.3)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    barrier()
    phase = np.zeros(5)
    with torch.cuda.stream(stream):
        e0.record(stream)
        for _ in range(args.steps):
            step_device()
            st.synchronize()
            phase += st.last_timings()[:5]
        e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    stop.set()
    th.join(timeout=3)
    barrier()
    t = torch.tensor([ms], dtype=torch.float64, device="cuda")
    if ws > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    ms_max = float(t.item())
    value = ws * nk * args.steps / (ms_max * 1e-3)
    phase /= max(args.steps, 1)

    # ---- the same batch replayed as one captured CUDA graph (no host work,
    # no synchronisation between steps)
    graph = st.graph(ngp, d_ig.data_ptr(), d_vg.data_ptr(), hp, op)
    for _ in range(args.warmup):
        graph.launch()
    st.synchronize()
    torch.cuda.synchronize()
    barrier()
    with torch.cuda.stream(stream):
        e0.record(stream)
        for _ in range(args.steps):
            graph.launch()
        e1.record(stream)
    st.synchronize()
    torch.cuda.synchronize()
    t = torch.tensor([e0.elapsed_time(e1)], dtype=torch.float64, device="cuda")
    if ws > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    graph_ms = float(t.item())
    graph.close()

    # ---- the interstitial gather alone (hmlistln + olpistln on the 27 H/O pairs),
    # HBM-bound: 32 N(N+1) bytes per k-point (read + write of the upper H and O)
    def gather_step():
        st.interstitial_batched_device(3, ngp, d_ig.data_ptr(), d_vg.data_ptr(), hp, op, nmat)
    for _ in range(args.warmup):
        gather_step()
    st.synchronize()
    torch.cuda.synchronize()
    with torch.cuda.stream(stream):
        e0.record(stream)
        for _ in range(args.steps):
            gather_step()
        e1.record(stream)
    st.synchronize()
    torch.cuda.synchronize()
    gather_ms = e0.elapsed_time(e1) / args.steps
    gather_bytes = sum(32.0 * n * (n + 1) for n in ngp)

    # ---- muffin-tin integral generation (hmlint), once per SCF iteration
    hml = None if args.skip_hmlint else hmlint_leg(args, st, s, stream, torch)

    # ---- real-time TDDFT Hamiltonian update of the same k-points
    rtl = None if args.skip_rttddft else rttddft_leg(args, st, stream, torch, ngp, nmat, d_ig, d_vg, hp, op,
                                                     step_device, s, gks)

    # ---- setup + device eigen-solve through the host entry point (only the
    # lowest 40 eigenpairs come back; the consumer solvewithlapack replaced)
    solve_value = None
    if not args.skip_e2e:
        nst = 40
        for _ in range(2):
            st.setup_and_solve(gks, nst)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        nrep = max(1, args.steps // 2)
        for _ in range(nrep):
            st.setup_and_solve(gks, nst)
        solve_value = ws * nk * nrep / (time.perf_counter() - t0)

    # ---- end to end through the host-pointer entry point
    e2e_modes = None
    if args.skip_e2e:
        e2e_value, h2d, d2h = None, 0, 0
    else:
        e2e_value, h2d, d2h = _e2e(args, st, stream, ig, vg, ngp, nmat, ws, barrier)
    if not args.skip_e2e and getattr(args, "e2e_modes", True):
        e2e_modes = {
            "pinned_direct": _e2e(args, st, stream, ig, vg, ngp, nmat, ws, barrier, "direct")[0],
            "pinned_packed": _e2e(args, st, stream, ig, vg, ngp, nmat, ws, barrier, "packed")[0],
            "pinned_upper": _e2e(args, st, stream, ig, vg, ngp, nmat, ws, barrier, "upper")[0],
            "pageable_direct": _e2e(args, st, stream, ig, vg, ngp, nmat, ws, barrier, "direct", False)[0],
            "pageable_packed": _e2e(args, st, stream, ig, vg, ngp, nmat, ws, barrier, "packed", False)[0],
        }

    # ---- split precision: its error against the native FP64 path on every
    # k-point of the batch (H and O on the device, Frobenius), the lowest 40
    # generalized eigenvalues of each by the device eigen-solve of both
    # paths, and the FP64 path's own device-resident rate for comparison
    accuracy, fp64_value = None, None
    if args.precision != "fp64":
        st.setup_batched_device(ngp, d_ig.data_ptr(), d_vg.data_ptr(), hp, op)
        st.synchronize()
        h_oz = [t.clone() for t in d_h]
        o_oz = [t.clone() for t in d_o]
        ev_oz, _ = st.setup_and_solve(gks, 40)
        st.set_precision("fp64")
        for _ in range(2):
            step_device()
        st.synchronize()
        torch.cuda.synchronize()
        barrier()
        with torch.cuda.stream(stream):
            e0.record(stream)
            for _ in range(args.steps):
                step_device()
            st.synchronize()
            e1.record(stream)
        torch.cuda.synchronize()
        t = torch.tensor([e0.elapsed_time(e1)], dtype=torch.float64, device="cuda")
        if ws > 1:
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
        fp64_value = ws * nk * args.steps / (float(t.item()) * 1e-3)
        fro_h = [_rel_fro_dev(a, b) for a, b in zip(h_oz, d_h)]
        fro_o = [_rel_fro_dev(a, b) for a, b in zip(o_oz, d_o)]
        del h_oz, o_oz
        ev_64, _ = st.setup_and_solve(gks, 40)
        dev = np.abs(ev_oz - ev_64)                        # (40, nk)
        accuracy = {
            "against": "native FP64 GPU path (itself within 1e-14 of the CPU oracle), all %d k-points" % nk,
            "eigen_solver": "exs_setup_and_solve_batched (cuSOLVER zhegvdx, lowest 40) on both paths",
            "rel_fro_H_max": float(max(fro_h)), "rel_fro_O_max": float(max(fro_o)),
            "max_abs_eig_dev_lowest40_Ha": float(dev.max()),
            "max_abs_eig_dev_per_k_Ha": [float(x) for x in dev.max(axis=0)],
            "max_rel_eig_dev_lowest40": float(np.max(dev / np.maximum(1.0, np.abs(ev_64)))),
            "lowest_eigenvalue_Ha": float(ev_64.min()),
            "gate_abs_1e-8_Ha": bool(dev.max() <= 1e-8),
        }

    # ---- the adjoint of one k-point (FP64 in either mode)
    adj = None if getattr(args, "skip_adjoint", False) else adjoint_leg(st, s, gks[0], torch)

    if rank == 0:
        fl = main_flops(s, gks)
        main_ms = phase[2]
        peak64 = _measured_fp64_peak(torch)
        achieved = fl / (main_ms * 1e-3) / 1e12
        if args.precision != "fp64":
            ops = ozaki_int8_ops(s, gks, products, ho_tile_cols(args.precision, tuned))
            peak8 = _measured_int8_peak(torch)
            a8 = ops / (main_ms * 1e-3) / 1e12
            roof = {"bound": "tensor", "kernel": ho_kernel(args.precision, tuned),
                    "achieved": a8, "peak": peak8, "unit": "TOP/s (int8)", "frac": a8 / peak8,
                    "peak_source": "cuBLASLt int8 GEMM 8192^3 (torch._int_mm) measured in this run",
                    "int8_ops_per_step": ops, "traffic": profiled_traffic_per_k(args.precision, tuned) * nk,
                    "traffic_note": "bytes per launch: ncu dram__bytes_read+write of a 2 k-point capture scaled "
                                    "by k-points; algorithmic %.3g" % main_bytes(s, gks, args.precision, planes),
                    "fp64_equivalent": {"achieved": achieved, "peak": peak64, "unit": "TFLOP/s",
                                        "frac": achieved / peak64,
                                        "peak_source": "cuBLAS DGEMM 8192^3 measured in this run"}}
        else:
            roof = {"bound": "tensor", "kernel": "zgemm_dmma_kernel<EPI_HAM>+<EPI_OVL> (MT contraction)",
                    "achieved": achieved, "peak": peak64, "unit": "TFLOP/s", "frac": achieved / peak64,
                    "peak_source": "cuBLAS DGEMM 8192^3 measured in this run (no FP64 entry in "
                                   "MEASURED_PEAKS.json)",
                    "algorithmic_flops_per_step": fl, "traffic": PROFILED_DRAM_BYTES_PER_K["fp64"] * nk,
                    "traffic_note": "bytes per step of <1>+<2>: ncu dram__bytes_read+write of a 6 k-point "
                                    "capture scaled by k-points; algorithmic %.3g" % main_bytes(s, gks, "fp64", 0)}
        clocks = _clock_summary(rows, local)
        cpu_v, cpu_n, cpu_dt = (None, 0, 0.0) if args.skip_cpu else cpu_sample(s, gks, budget_s=12.0)
        out = {
            "metric": METRIC, "value": value, "unit": "setups/s", "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None,
            "dtype": dtype_text if args.precision != "fp64" else "f64", "data": "synthetic",
            "config": {"workload": WORKLOAD, "k_per_step": nk, "ngp": [min(ngp), max(ngp)],
                       "nmat": [min(nmat), max(nmat)],
                       "kernel_config": tuned,
                       "precision": prec_text if args.precision != "fp64" else "fp64 (DMMA)",
                       "l2": "working set > 126 MB L2 (A/B planes 63 MB and H/O 48 MB per k-point), no flush"},
            "e2e": None if e2e_value is None else {
                "value": e2e_value, "unit": "setups/s", "h2d_bytes_per_step": int(h2d),
                "d2h_bytes_per_step": int(d2h), "host_copy_mode": "auto (pinned outputs)",
                "by_copy_mode": e2e_modes},
            "phases_ms_per_step": {"match": phase[0], "h_a_A": phase[1], "mt_contraction": phase[2],
                                   "lo_blocks": phase[3], "total": phase[4]},
            "graph_replay": {"value": ws * nk * args.steps / (graph_ms * 1e-3), "unit": "setups/s",
                             "ms_per_step": graph_ms / args.steps,
                             "note": "same batch captured once (exs_graph_create) and replayed"},
            "roofline": roof,
            "setup_and_solve": None if solve_value is None else {
                "value": solve_value, "unit": "k-points/s", "nstfv": 40,
                "note": "exs_setup_and_solve_batched: setup + cuSOLVER zhegvdx (lowest 40 pairs) on the device, "
                        "eigenpairs to the host; wall clock"},
            "interstitial_gather": {
                "kernel": "interstitial_kernel (exs_interstitial_batched_device: hmlistln + olpistln, 27 k-points "
                          "in one launch)",
                "ms_per_step": gather_ms, "bytes_per_step": gather_bytes,
                "achieved": gather_bytes / (gather_ms * 1e-3) / 1e9, "unit": "GB/s",
                "peak": _hbm_peak(), "frac": gather_bytes / (gather_ms * 1e-3) / 1e9 / _hbm_peak(),
                "peak_source": "MEASURED_PEAKS.json hbm_gbs (measured)"},
            "cpu_baseline": None if cpu_v is None else {
                "value": cpu_v, "unit": "setups/s", "cores": os.cpu_count(), "kind": "port",
                "sample": f"{cpu_n} k-points of the 27-k set in {cpu_dt:.1f} s by the FP64 CPU "
                          "restatement (C + OpenMP + OpenBLAS zgemm)"},
            "clocks": clocks,
            "gpu_launches": launches_per_setup(args.precision) * args.steps,
            "setup_flops_per_step": setup_flops(s, gks),
            "accuracy": accuracy,
            "fp64_path_value": fp64_value,
            "adjoint": adj,
            "hmlint": hml,
            "rttddft_updateham": rtl,
        }
        if emit:
            print(json.dumps(out), flush=True)
    st.set_stream(None)
    st.close()
    if ws > 1:
        dist.barrier()
        dist.destroy_process_group()
    return 0 if emit else (out if rank == 0 else None)


WORKLOAD_216 = ("si_cube216 216-atom Si (3x3x3 supercell of the 8-atom cube, a = 30.78), Gamma + 3 k, "
                "rgkmax 8, lmaxapw 8, APW order 2, 1 lo per l<=2")


def _rel_fro_dev(a, b, chunk=1 << 27):
    num = den = 0.0
    for i in range(0, a.numel(), chunk):
        x, y = a[i:i + chunk], b[i:i + chunk]
        num += float(((x - y) ** 2).sum())
        den += float((y ** 2).sum())
    return (num / den) ** 0.5


def _host(t, n):
    """The first n doubles of a device tensor, on the host (pageable)."""
    return t[:n].cpu()


def _rel_fro_host(h, d, chunk=1 << 27):
    """||h - d|| / ||d|| for a host tensor h and a device tensor d of the same length."""
    num = den = 0.0
    for i in range(0, h.numel(), chunk):
        x = h[i:i + chunk].cuda(non_blocking=False)
        y = d[i:i + chunk]
        num += float(((x - y) ** 2).sum())
        den += float((y ** 2).sum())
    return (num / den) ** 0.5


def _lowest_generalized(solver, h, o, m, nev, torch):
    """The lowest nev eigenvalues of H x = e O x for za(m, m) matrices held as
    host tensors of 2 m^2 doubles, by the library's device eigen-solve
    (exs_solve_batched_device: cuSOLVER zhegvdx, index range 1..nev, values
    only) on a context `solver` that only lends its solver handles."""
    import ctypes
    H, O_ = h.cuda(), o.cuda()
    ev = torch.zeros(nev, dtype=torch.float64, device="cuda")
    nmat = (ctypes.c_int * 1)(m)
    hp = (ctypes.c_void_p * 1)(H.data_ptr())
    op = (ctypes.c_void_p * 1)(O_.data_ptr())
    solver._check(solver.lib.exs_solve_batched_device(solver.ctx, 1, nmat, hp, op, nev,
                                                      ctypes.c_void_p(ev.data_ptr()), None, m))
    w = ev.cpu().numpy()
    del H, O_
    torch.cuda.empty_cache()
    return w


def _lowest_generalized_reduced(h, o, m, nev, torch):
    """The lowest nev eigenvalues of H x = e O x by a Cholesky reduction
    (cuSOLVER potrf and two triangular solves, through torch) to the dense
    Hermitian C = L^-1 H L^-H and its eigenvalues through torch's MAGMA
    backend (hybrid host/device), for orders where cuSOLVER's dense
    eigen-solvers return an invalid-value status.  The za(m, m) host tensors
    read as the transposes conj(H), conj(O): the same eigenvalues."""
    H = h.cuda().view(torch.complex128).view(m, m)
    L = torch.linalg.cholesky(o.cuda().view(torch.complex128).view(m, m))
    X = torch.linalg.solve_triangular(L, H, upper=False)                   # L^-1 H
    del H
    C = torch.linalg.solve_triangular(L, X.mH.contiguous(), upper=False)   # L^-1 H L^-H
    del X, L
    torch.cuda.empty_cache()
    prev = torch.backends.cuda.preferred_linalg_library()
    torch.backends.cuda.preferred_linalg_library("magma")
    try:
        w = torch.linalg.eigvalsh(C)[:nev].cpu().numpy()
    finally:
        torch.backends.cuda.preferred_linalg_library(prev)
    del C
    torch.cuda.empty_cache()
    return w


def _ritz_compare(pencils, base, m, nev, torch, nx=64):
    """Eigenvalue deviations between pencils (H, O) free of the dense
    solver's own rounding: the lowest nx eigenvectors X of pencils[base]
    (Cholesky reduction, dense eigen-solve with vectors through torch's MAGMA
    backend, X = L^-H Y), then the Ritz values of every pencil on span(X)
    (nx x nx generalized problems).  For pencils[base] they are its
    eigenvalues; for another pencil they differ from its eigenvalues by the
    square of the residual over the gap (second order in the ~1e-13
    difference of the matrices).  Returns (lowest nev eigenvalues of the
    dense solve, [lowest nev Ritz values of each pencil])."""
    c128 = torch.complex128
    prev = torch.backends.cuda.preferred_linalg_library()
    h64, o64 = pencils[base]
    H = h64.cuda().view(c128).view(m, m)
    L = torch.linalg.cholesky(o64.cuda().view(c128).view(m, m))
    X1 = torch.linalg.solve_triangular(L, H, upper=False)
    del H
    C = torch.linalg.solve_triangular(L, X1.mH.contiguous(), upper=False)
    del X1
    torch.cuda.empty_cache()
    torch.backends.cuda.preferred_linalg_library("magma")
    try:
        w, Y = torch.linalg.eigh(C)
    finally:
        torch.backends.cuda.preferred_linalg_library(prev)
    del C
    Y = Y[:, :nx].contiguous()
    w = w[:nev].cpu().numpy()
    torch.cuda.empty_cache()
    X = torch.linalg.solve_triangular(L.mH.contiguous(), Y, upper=True)     # L^-H Y
    del L, Y
    torch.cuda.empty_cache()

    def ritz(h, o):
        A = h.cuda().view(c128).view(m, m)
        Hs = X.mH @ (A @ X)
        del A
        B = o.cuda().view(c128).view(m, m)
        Os = X.mH @ (B @ X)
        del B
        torch.cuda.empty_cache()
        Hs = 0.5 * (Hs + Hs.mH)
        Os = 0.5 * (Os + Os.mH)
        Ls = torch.linalg.cholesky(Os)
        Cs = torch.linalg.solve_triangular(Ls, torch.linalg.solve_triangular(Ls, Hs, upper=False).mH, upper=False)
        return torch.linalg.eigvalsh(0.5 * (Cs + Cs.mH))[:nev].cpu().numpy()
    th = [ritz(h, o) for h, o in pencils]
    del X
    torch.cuda.empty_cache()
    return w, th


def _progress(msg):
    print("[bench] %s" % msg, file=sys.stderr, flush=True)


def adjoint_recipe(nmat, seed=3, nst=40):
    """The force-check states: nst orthonormal complex vectors (QR of a
    Gaussian, seed 3), w = 2, eps ~ U[-0.5, 0.5] Ha."""
    rng = np.random.default_rng(seed)
    c, _ = np.linalg.qr(rng.standard_normal((nmat, nst)) + 1j * rng.standard_normal((nmat, nst)))
    eps = rng.uniform(-0.5, 0.5, nst)
    return np.asfortranarray(c), np.full(nst, 2.0), eps


def adjoint_flops(sys_, gk, nst):
    """Algorithmic flops of the factored adjoint: U_q = A_a C (q = 0..3), h_a U_q,
    and the two N x N rank-nst products P and Q (8 flops per complex MAC)."""
    b = sys_.basis
    K = sum(b.napw_atom(a) for a in range(sys_.natmtot))
    m2 = sum(b.napw_atom(a) ** 2 for a in range(sys_.natmtot))
    n = gk.ngp
    return 4 * 8.0 * K * n * nst + 4 * 8.0 * m2 * nst + 2 * 8.0 * n * n * nst


def adjoint_leg(st, sys_, gk, torch, reps=3):
    """exs_adjoint (dL/dtau, dL/dV, dL/dh_a) on one k-point with the force-check
    states, wall clock of the synchronous call (uploads of the states included)."""
    c, w, eps = adjoint_recipe(sys_.nmat(gk))
    out = st.adjoint(gk, c, w, eps, dveffig=True, dh=True)       # warm-up (work space, output arrays)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(reps):                                         # the caller's arrays, as a Fortran caller passes them
        dtau, _, _ = st.adjoint(gk, c, w, eps, dveffig=True, dh=True, out=out)
    dt = (time.perf_counter() - t0) / reps
    fl = adjoint_flops(sys_, gk, c.shape[1])
    return {"ms": dt * 1e3, "k_points_per_s": 1.0 / dt, "states": int(c.shape[1]),
            "flops": fl, "achieved_tflops": fl / dt / 1e12,
            "max_abs_dL_dtau": float(np.max(np.abs(dtau))),
            "note": "exs_adjoint: dL/dtau (= -F_IBS), dL/dV(G), dL/dh_a for 40 orthonormal states, w = 2, "
                    "eps ~ U[-0.5, 0.5] (seed 3); FP64 in either precision mode; wall clock of the call"}


def cpu_sample_216(sys_, gk, m_atoms=1, n_sub=3000):
    """The FP64 CPU restatement on a bounded sample of one 216-atom k-point:
    match and the H and O zgemm pairs (hamiltonsetup.f90:75-103,
    overlapsetup.f90:88-101) of m_atoms atoms, and hmlistln/olpistln over the
    first n_sub G+k; extrapolated linearly in atoms and by N(N+1) in G+k.
    Returns (extrapolated seconds per k-point, sample seconds)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import lapw_oracle as O
    from exciting_b200.crystal import gensfacgp
    lib = O.lib()
    b = sys_.basis
    n = gk.ngp
    t0 = time.perf_counter()
    # match for the sample atoms
    gpc = np.ascontiguousarray(gk.gpc)
    tpgpc = np.asfortranarray(gk.tpgpc)
    sf = np.asfortranarray(gensfacgp(gk.vgpc, sys_.crystal.atposc[:, :m_atoms]))
    apword = O._f(np.array(b.apword).T, np.int32)
    species = np.asarray(b.atom_species[:m_atoms], dtype=np.int32)
    apwalm = np.zeros((n, b.apwordmax, b.lmmaxapw, m_atoms), dtype=np.complex128, order="F")
    tail = np.asfortranarray(sys_.apwfr_tail[..., :m_atoms])
    lib.orc_match(n, n, O._p(gpc), O._p(tpgpc), O._p(sf), m_atoms, O._p(species), b.lmaxapw, b.apwordmax,
                  O._p(apword), O._p(O._f(sys_.rmt, np.float64)), sys_.crystal.omega, sys_.np_tail,
                  O._p(O._f(sys_.spr_tail, np.float64)), O._p(tail), O._p(apwalm))
    t_match = time.perf_counter() - t0
    # the zgemm pairs into full N x N accumulators, as the reference (beta = 1)
    import scipy.linalg.blas as blas
    h = np.zeros((n, n), dtype=np.complex128, order="F")
    t1 = time.perf_counter()
    for ias in range(m_atoms):
        apwi = np.asfortranarray(O._apwi(sys_, apwalm, n, ias))
        zm = blas.zgemm(1.0, np.asfortranarray(sys_.mt_aa[:, :, ias]), apwi)
        h = blas.zgemm(1.0, apwi, zm, beta=1.0, c=h, trans_a=2, overwrite_c=1)
        h = blas.zgemm(1.0, apwi, apwi, beta=1.0, c=h, trans_a=2, overwrite_c=1)    # the O pair, same cost
    t_pairs = time.perf_counter() - t1
    del h
    # hmlistln + olpistln over the first n_sub G+k
    ns = min(n_sub, n)
    gv = sys_.gv
    hs = np.zeros((ns, ns), dtype=np.complex128, order="F")
    os_ = np.zeros((ns, ns), dtype=np.complex128, order="F")
    ivg = O._f(gv.ivg, np.int32)
    ivgig = np.asfortranarray(gv.ivgig, dtype=np.int32)
    intgv = O._f(gv.intgv, np.int32)
    vgpc = O._f(gk.vgpc[:, :ns], np.float64)
    igpig = O._f(gk.igpig[:ns], np.int32)
    kinw = O._f(sys_.kinetic_weight, np.complex128)
    t2 = time.perf_counter()
    lib.orc_hmlistln_olpistln(ns, O._p(igpig), O._p(vgpc), ns, O._p(ivg), O._p(ivgig), O._p(intgv), gv.ngvec,
                              O._p(sys_.veffig), O._p(kinw), O._p(sys_.cfunig), None, 0, O._p(hs), O._p(os_))
    t_int = time.perf_counter() - t2
    scale_a = sys_.natmtot / m_atoms
    full = (t_match + t_pairs) * scale_a + t_int * (n * (n + 1.0)) / (ns * (ns + 1.0))
    return full, time.perf_counter() - t0


def e2e_large(st, gks, nlotot, mmax, torch, ne=2):
    """Setups/s through exs_setup_batched, one k-point per call: igpig/vgpc in
    from the host, H and O (13.6 GB each) back into pinned host memory."""
    hp = torch.empty(2 * mmax * mmax, dtype=torch.float64, pin_memory=True)
    op = torch.empty_like(hp, pin_memory=True)

    def views(g):     # za(nmat, nmat) of this k-point at the start of the pinned buffers
        m = g.ngp + nlotot
        return [(hp.numpy()[: 2 * m * m].view(np.complex128).reshape(m, m, order="F"),
                 op.numpy()[: 2 * m * m].view(np.complex128).reshape(m, m, order="F"))]
    st.setup_batched([gks[0]], out=views(gks[0]))          # warm-up
    t0 = time.perf_counter()
    for i in range(ne):
        g = gks[i % len(gks)]
        st.setup_batched([g], out=views(g))
    dt = time.perf_counter() - t0
    m0 = gks[0].ngp + nlotot
    return {"value": ne / dt, "unit": "setups/s", "h2d_bytes_per_step": int(gks[0].ngp * 16),
            "d2h_bytes_per_step": int(2 * 16 * m0 * m0), "host_copy_mode": "auto (pinned outputs)",
            "steps": ne, "note": "exs_setup_batched, one k-point per call: igpig/vgpc in, H and O (13.6 GB "
                                 "each) to pinned host memory; wall clock"}


def run_large(args):
    """The 216-atom cell, the default workload: one k-point per step (H and
    O are ~13.6 GB each), Gamma and the three other k-points in turn.  Timed:
    the split-precision setup (value), the native FP64 path, the adjoint, and
    the host-pointer entry point; accuracy at Gamma (Frobenius and the lowest
    40 generalized eigenvalues of both paths); the CPU restatement on a bounded
    sample; the 8-atom batch as a secondary leg.  With several ranks every
    rank times the split and FP64 legs and the adjoint; the accuracy,
    eigenvalue, CPU and 8-atom legs run in one-GPU runs only."""
    import torch
    import torch.distributed as dist
    from exciting_b200 import workloads as W
    from exciting_b200.fvsystem import Setup

    ws, rank = _dist()
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if ws > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=600), device_id=torch.device("cuda", local))
    s = W.si_cube216()
    gks_all = s.gksets()[: min(args.nk, 4)]
    # every rank sets up one k-point per step, starting at its own k-point (weak scaling)
    r0 = rank % len(gks_all)
    gks = gks_all[r0:] + gks_all[:r0]
    st = Setup(s, ngkmax=max(g.ngp for g in gks_all), max_batch=1)
    stream = torch.cuda.Stream()
    st.set_stream(stream.cuda_stream)
    ngkmax, nlotot = st.ngkmax, st.nlotot
    ig, vg = [], []
    for g in gks:
        a = np.zeros(ngkmax, dtype=np.int32)
        a[: g.ngp] = g.igpig
        b = np.zeros((ngkmax, 3))
        b[: g.ngp] = g.vgpc.T
        ig.append(torch.from_numpy(a).cuda())
        vg.append(torch.from_numpy(b).cuda())
    mmax = ngkmax + nlotot
    d_h = torch.empty(2 * mmax * mmax, dtype=torch.float64, device="cuda")
    d_o = torch.empty_like(d_h)

    def one(k):
        st.setup_batched_device([gks[k].ngp], ig[k].data_ptr(), vg[k].data_ptr(), [d_h.data_ptr()],
                                [d_o.data_ptr()])

    def timed(nsteps, nwarm, sample_clocks):
        for i in range(nwarm):
            one(i % len(gks))
            st.synchronize()
        rows, stop = [], threading.Event()
        th = None
        if sample_clocks:
            th = threading.Thread(target=_clock_sampler, args=(stop, rows), daemon=True)
            th.start()
            time.sleep(0.3)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        if ws > 1:
            dist.barrier()
        phase = np.zeros(5)
        with torch.cuda.stream(stream):
            e0.record(stream)
            for i in range(nsteps):
                one(i % len(gks))
                st.synchronize()
                phase += st.last_timings()[:5]
            e1.record(stream)
        torch.cuda.synchronize()
        stop.set()
        if th is not None:
            th.join(timeout=3)
        t = torch.tensor([e0.elapsed_time(e1)], dtype=torch.float64, device="cuda")
        if ws > 1:
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item()), phase / max(nsteps, 1), rows

    prec = args.precision if args.precision != "fp64" else "ozaki_mod"
    st.set_precision(prec, args.slices if prec == "ozaki" else args.moduli)
    args.precision = prec
    if args.kernel_config >= 0:
        st.set_kernel_config(args.kernel_config)
    # the library's default until a configuration is chosen: paced persistent two-SM residue tiles with moduli
    kcfg = args.kernel_config if args.kernel_config >= 0 else (10 if prec == "ozaki_mod" else 0)
    planes, products, dtype_text, prec_text = split_scheme(args, s)
    ms, phase, rows = timed(args.steps, args.warmup, True)
    value = ws * args.steps / (ms * 1e-3)
    _progress("split: %.4f setups/s, phases %s" % (value, list(np.round(phase, 2))))
    m0 = gks[0].ngp + nlotot
    nf = len(gks)
    fp64_value, phase64, acc, h8, h16 = None, np.zeros(5), None, None, None
    if not args.skip_fp64:
        # ---- Gamma in split precision, kept on the host for the comparison (one GPU only: 27 GB per pencil)
        if ws == 1:
            one(0)
            st.synchronize()
            h8, o8 = _host(d_h, 2 * m0 * m0), _host(d_o, 2 * m0 * m0)
        # ---- the native FP64 path: a few stated steps (one per k-point), every rank
        st.set_precision("fp64")
        ms64, phase64, _ = timed(nf, 1, False)
        fp64_value = ws * nf / (ms64 * 1e-3)
        _progress("fp64: %.4f setups/s, phases %s" % (fp64_value, list(np.round(phase64, 2))))
        if ws == 1:
            one(0)
            st.synchronize()
            acc = {"against": "native FP64 GPU path, Gamma, whole H and O",
                   "rel_fro_H": _rel_fro_host(h8, d_h[: 2 * m0 * m0]),
                   "rel_fro_O": _rel_fro_host(o8, d_o[: 2 * m0 * m0])}
            h64, o64 = _host(d_h, 2 * m0 * m0), _host(d_o, 2 * m0 * m0)
        if not args.skip_eig and ws == 1 and prec == "ozaki_mod" and args.moduli != 16:
            # ---- a third Gamma pencil, the split path at its widest plan (16 moduli, 52-bit operands):
            # the eigenvalue leg separates the split path's own error from the FP64 path's rounding
            try:
                st.set_precision("ozaki_mod", 16)
                one(0)
                st.synchronize()
                acc.update({"rel_fro_H_16_moduli_vs_fp64": _rel_fro_host(h64, d_h[: 2 * m0 * m0]),
                            "rel_fro_H_vs_16_moduli": _rel_fro_host(h8, d_h[: 2 * m0 * m0]),
                            "rel_fro_O_vs_16_moduli": _rel_fro_host(o8, d_o[: 2 * m0 * m0])})
                h16, o16 = _host(d_h, 2 * m0 * m0), _host(d_o, 2 * m0 * m0)
            except Exception as e:      # reported, not fatal
                acc["moduli_16_error"] = str(e)[:300]
    del d_h, d_o
    torch.cuda.empty_cache()
    # ---- end to end through the host-pointer entry point (pinned H and O, 13.6 GB each per k-point)
    _progress("accuracy: %s" % json.dumps(acc))
    e2e = None
    if not args.skip_e2e and rank == 0:
        try:
            st.set_precision(prec, args.slices if prec == "ozaki" else args.moduli)
            e2e = e2e_large(st, gks, nlotot, mmax, torch)
        except Exception as e:      # reported, not fatal
            e2e = {"error": str(e)[:300]}
        _progress("e2e: %s" % json.dumps(e2e))
    # ---- the adjoint at Gamma (FP64 in either mode)
    adj = None
    if not args.skip_adjoint:
        try:
            adj = adjoint_leg(st, s, gks[0], torch)
        except Exception as e:      # reported, not fatal
            adj = {"error": str(e)[:300]}
        _progress("adjoint: %s" % json.dumps(adj))
    clocks = _clock_summary(rows, local)
    st.set_stream(None)
    st.close()
    torch.cuda.empty_cache()
    # ---- eigenvalues of both Gamma pairs
    if args.dense_eig and not args.skip_eig and h8 is not None and rank == 0:
        t0 = time.perf_counter()
        how = "exs_solve_batched_device (cuSOLVER zhegvdx, lowest 40, values only) on each path's H and O"
        w8 = w64 = None
        try:
            solver = Setup(W.si_fcc("text"))
            try:
                w8 = _lowest_generalized(solver, h8, o8, m0, 40, torch)
                w64 = _lowest_generalized(solver, h64, o64, m0, 40, torch)
            finally:
                solver.close()
        except Exception as e:      # cuSOLVER's dense solvers refuse this order: the reduced form
            acc["cusolver_error"] = str(e)[:200]
            how = ("Cholesky reduction (cuSOLVER potrf + triangular solves) and the dense Hermitian eigen-solve "
                   "through torch's MAGMA backend, lowest 40 of each path")
            try:
                w8 = _lowest_generalized_reduced(h8, o8, m0, 40, torch)
                w64 = _lowest_generalized_reduced(h64, o64, m0, 40, torch)
            except Exception as e2:      # reported, not fatal: the timing legs stand
                acc["eigen_solver_error"] = str(e2)[:300]
        if w8 is not None and w64 is not None:
            acc.update({"eigen_solver": how, "eig_solve_s": time.perf_counter() - t0,
                        "max_abs_eig_dev_lowest40_dense_Ha": float(np.max(np.abs(w8 - w64))),
                        "lowest_eigenvalue_Ha": float(w64[0])})
            acc["dense_w64"] = w64
    if not args.skip_eig and h8 is not None and rank == 0:
        # the comparison free of the dense solver's rounding: Ritz values of every pencil on one subspace
        try:
            t1 = time.perf_counter()
            pencils = [(h8, o8), (h64, o64)] + ([(h16, o16)] if h16 is not None else [])
            wd, th = _ritz_compare(pencils, 1, m0, 40, torch)
            t8, t64 = th[0], th[1]
            dev = float(np.max(np.abs(t8 - t64)))
            acc.update({"ritz": "Ritz values of each pencil on the FP64 pencil's lowest 64 eigenvectors "
                                "(dense MAGMA eigen-solve with vectors); second order in the H/O differences",
                        "ritz_s": time.perf_counter() - t1,
                        "max_abs_eig_dev_lowest40_Ha": dev,
                        "fp64_ritz_vs_dense_Ha": float(np.max(np.abs(t64 - wd))),
                        "lowest_eigenvalue_Ha": float(wd[0]),
                        "gate_abs_1e-8_Ha": {"vs_fp64_path": bool(dev <= 1e-8)}})
            if h16 is not None:
                # the widest split plan (52-bit operands, products accumulated exactly, one rounding) as
                # the reference: the split path's own error, and the FP64 path's accumulation rounding
                d16 = float(np.max(np.abs(t8 - th[2])))
                acc.update({"exact_accumulation_reference": "split path with 16 moduli: FP64 operands rounded "
                                                            "to 52 bits below their column norms, products "
                                                            "exact in integers (CRT), one rounding per element",
                            "max_abs_eig_dev_lowest40_vs_exact_accumulation_Ha": d16,
                            "fp64_path_vs_exact_accumulation_Ha": float(np.max(np.abs(t64 - th[2])))})
                acc["gate_abs_1e-8_Ha"]["vs_exact_accumulation"] = bool(d16 <= 1e-8)
            w64 = acc.pop("dense_w64", None)
            if w64 is not None:
                acc["dense_solver_repeat_vs_first_Ha"] = float(np.max(np.abs(wd - w64)))
        except Exception as e:      # reported, not fatal
            acc["ritz_error"] = str(e)[:300]
        _progress("eigenvalues: %s" % json.dumps({k: v for k, v in acc.items()
                                                  if "eig" in k or "moduli" in k or "accumulation" in k or "gate" in k}))
    if acc is not None:
        acc.pop("dense_w64", None)
    if h8 is not None:
        del h8, o8, h64, o64
    if h16 is not None:
        del h16, o16
    if ws > 1:
        dist.barrier()
    if rank == 0:
        ops = ozaki_int8_ops(s, gks_all, products, ho_tile_cols(prec, kcfg)) / len(gks_all)   # per k-point
        fl = main_flops(s, gks_all) / len(gks_all)
        peak8 = _measured_int8_peak(torch)
        peak8s, clk8s = _measured_int8_sustained(torch)
        peak64 = _measured_fp64_peak(torch)
        mt_ms = phase[2]
        a8 = ops / (mt_ms * 1e-3) / 1e12
        cpu = None
        if not args.skip_cpu and ws == 1:
            try:
                cpu_sample_216(s, gks_all[0], 1, 1000)                      # warm-up (libraries, pages)
                full, dt = cpu_sample_216(s, gks_all[0], 2, 3000)
                cpu = {"value": 1.0 / full, "unit": "setups/s", "cores": os.cpu_count(), "kind": "port",
                       "sample": "Gamma: match and the H and O zgemm pairs of 2 of 216 atoms plus "
                                 "hmlistln/olpistln over 3000 of %d G+k by the FP64 CPU restatement (C + "
                                 "OpenBLAS zgemm, %.1f s), extrapolated linearly in atoms and by N(N+1) in G+k"
                                 % (gks_all[0].ngp, dt)}
            except Exception as e:      # reported, not fatal
                cpu = {"error": str(e)[:300]}
            _progress("cpu: %s" % json.dumps(cpu))
        sub = None
        if not args.skip_cube8 and ws == 1:
            try:
                sub = run_ours(argparse.Namespace(**{**vars(args), "steps": 10, "warmup": 3, "nk": 27,
                                                     "skip_cpu": True, "skip_hmlint": True, "skip_rttddft": True,
                                                     "skip_e2e": True, "e2e_modes": False}), emit=False)
            except Exception as e:      # reported, not fatal
                sub = {"error": str(e)[:300]}
        out = {
            "metric": METRIC, "value": value, "unit": "setups/s", "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": dtype_text,
            "data": "synthetic",
            "config": {"workload": WORKLOAD_216, "k_per_step": 1,
                       "kpoints": "Gamma, (1/2,0,0), (1/2,1/2,0), (1/2,1/2,1/2) in turn, one per step",
                       "ngp": [min(g.ngp for g in gks_all), max(g.ngp for g in gks_all)],
                       "nmat": [min(g.ngp for g in gks_all) + nlotot, max(g.ngp for g in gks_all) + nlotot],
                       "precision": prec_text, "kernel_config": kcfg,
                       "l2": "working set (A/B planes 30 GB, %d int8 planes of 4 arrays, H/O 27 GB) far above "
                             "L2, no flush" % planes},
            "e2e": e2e,
            "phases_ms_per_step": {"match": phase[0], "h_a_A": phase[1], "mt_contraction": phase[2],
                                   "lo_blocks": phase[3], "total": phase[4]},
            "roofline": {"bound": "tensor", "kernel": ho_kernel(prec, kcfg),
                         "achieved": a8, "peak": peak8s, "unit": "TOP/s (int8)", "frac": a8 / peak8s,
                         "peak_source": "cuBLASLt int8 GEMM 8192^3 (torch._int_mm) back to back for 4 s in this "
                                        "run (sustained, under the power cap: the H/O kernel runs for seconds)",
                         "peak_burst": peak8, "frac_of_burst": a8 / peak8, "peak_sustained_clocks": clk8s,
                         **_int8_from_bf16_peaks(a8),
                         "int8_ops_per_step": ops, "traffic": PROFILED_DRAM_BYTES_216.get(kcfg),
                         "traffic_note": "bytes per launch of the residue kernel: ncu dram__bytes_read+write of "
                                         "one full-size launch (one pass); algorithmic %.3g (residue planes read "
                                         "once, residues written once)" % residue_bytes(s, gks_all[0], planes),
                         "fp64_equivalent": {"achieved": fl / (mt_ms * 1e-3) / 1e12, "peak": peak64,
                                             "unit": "TFLOP/s", "frac": fl / (mt_ms * 1e-3) / 1e12 / peak64}},
            "cpu_baseline": cpu,
            "clocks": clocks,
            "gpu_launches": launches_per_setup(prec) * args.steps,
            "setup_flops_per_step": setup_flops(s, gks_all) / len(gks_all),
            "accuracy": acc,
            "fp64_path_value": fp64_value,
            "fp64_steps": nf,
            "fp64_phases_ms_per_step": {"match": phase64[0], "h_a_A": phase64[1], "mt_contraction": phase64[2],
                                        "lo_blocks": phase64[3], "total": phase64[4]},
            "speedup_split_vs_fp64": None if fp64_value is None else value / fp64_value,
            "adjoint": adj,
            "with_adjoint": None if (adj is None or fp64_value is None or "ms" not in adj) else {
                "split_setups_per_s": 1.0 / (1.0 / value + adj["ms"] * 1e-3),
                "fp64_setups_per_s": 1.0 / (1.0 / fp64_value + adj["ms"] * 1e-3),
                "note": "setup + adjoint per k-point, both paths (the adjoint runs in FP64 in either)"},
            "cube8": sub,
        }
        print(json.dumps(out), flush=True)
    if ws > 1:
        dist.barrier()
        dist.destroy_process_group()
    return 0


WORKLOAD_CELLS = ("si_fcc_random x256: independent 2-atom fcc Si cells, a ~ U[9.8, 10.8], rgkmax in {6,7,8,9} "
                  "(seed 4+i), lmaxapw 8, Gamma point each; one context per cell, all cells in one CUDA graph")


def run_cells(args):
    """The uneven-size batch: 256 independent cells, one context each, set up
    together by one multi-context CUDA graph per step."""
    import torch
    from exciting_b200 import workloads as W
    from exciting_b200.fvsystem import Setup, multi_graph

    ws, rank = _dist()
    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    ncell = min(args.nk, 256) if args.nk != 27 else 256
    cells = [W.si_fcc_random(i) for i in range(ncell)]
    stream = torch.cuda.Stream()
    setups, batches, keep, tuned = [], [], [], []
    for s in cells:
        gk = s.gkset(s.kpoints[0])
        st = Setup(s, max_batch=1)
        st.set_precision(args.precision, args.slices if args.precision != "ozaki_mod" else args.moduli)
        ig = np.zeros(st.ngkmax, dtype=np.int32)
        ig[: gk.ngp] = gk.igpig
        vg = np.zeros((st.ngkmax, 3))
        vg[: gk.ngp] = gk.vgpc.T
        m = gk.ngp + st.nlotot
        t = (torch.from_numpy(ig).cuda(), torch.from_numpy(vg).cuda(),
             torch.empty(2 * m * m, dtype=torch.float64, device="cuda"),
             torch.empty(2 * m * m, dtype=torch.float64, device="cuda"), gk.ngp)
        keep.append(t)
        b = ([gk.ngp], t[0].data_ptr(), t[1].data_ptr(), [t[2].data_ptr()], [t[3].data_ptr()])
        tuned.append(st.autotune(*b))
        setups.append(st)
        batches.append(b)
    setups[0].set_stream(stream.cuda_stream)
    g = multi_graph(setups, batches)
    for _ in range(args.warmup):
        g.launch()
    g.synchronize()
    rows, stop = [], threading.Event()
    th = threading.Thread(target=_clock_sampler, args=(stop, rows), daemon=True)
    th.start()
    time.sleep(0.3)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    with torch.cuda.stream(stream):
        e0.record(stream)
        for _ in range(args.steps):
            g.launch()
        e1.record(stream)
    g.synchronize()
    torch.cuda.synchronize()
    stop.set()
    th.join(timeout=3)
    ms = e0.elapsed_time(e1)
    # the same cells one after another through the device entry point (no graph)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for st, b in zip(setups, batches):
        st.setup_batched_device(*b)
    for st in setups:
        st.synchronize()
    seq_ms = (time.perf_counter() - t0) * 1e3
    g.close()
    if rank == 0:
        ngp = [t[4] for t in keep]
        cpu_v, cpu_n, cpu_dt = (None, 0, 0.0)
        if not args.skip_cpu:
            sys.path.insert(0, os.path.join(ROOT, "oracle"))
            import lapw_oracle as O
            t0 = time.perf_counter()
            for s in cells:
                O.hamiltonandoverlapsetup(s, s.gkset(s.kpoints[0]))
                cpu_n += 1
                if time.perf_counter() - t0 > 10.0:
                    break
            cpu_dt = time.perf_counter() - t0
            cpu_v = cpu_n / cpu_dt
        out = {
            "metric": METRIC, "value": ncell * args.steps / (ms * 1e-3), "unit": "setups/s", "n_gpus": ws,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None,
            "dtype": {"ozaki": "i8 slices, f64 recombination", "fp64": "f64"}.get(
                args.precision, "i8 residues modulo coprime moduli (per-cell count), CRT recombination"),
            "data": "synthetic",
            "config": {"workload": WORKLOAD_CELLS, "cells_per_step": ncell, "ngp": [min(ngp), max(ngp)],
                       "precision": args.precision, "kernel_configs": sorted(set(tuned)),
                       "l2": "all cells' working set ~3 GB > L2, no flush"},
            "sequential_device_calls_ms": seq_ms,
            "e2e": None,
            "cpu_baseline": None if cpu_v is None else {
                "value": cpu_v, "unit": "setups/s", "cores": os.cpu_count(), "kind": "port",
                "sample": f"{cpu_n} cells by the FP64 CPU restatement in {cpu_dt:.1f} s"},
            "clocks": _clock_summary(rows, 0),
            "gpu_launches": launches_per_setup(args.precision) * ncell * args.steps,
        }
        print(json.dumps(out), flush=True)
    for st in setups:
        st.close()
    return 0


def run_hmlint(args):
    """The muffin-tin integral leg alone (one GPU) on the 8- or 216-atom cell:
    a context with a token G+k size (the integrals need no G+k set)."""
    import torch
    from exciting_b200 import workloads as W
    from exciting_b200.fvsystem import Setup
    ws, rank = _dist()
    if rank != 0:
        return 0
    s = W.si_cube216() if args.workload == "cube216" else W.si_cube8()
    st = Setup(s, ngkmax=64, max_batch=1)
    stream = torch.cuda.Stream()
    st.set_stream(stream.cuda_stream)
    leg = hmlint_leg(args, st, s, stream, torch)
    out = {"metric": "muffin-tin integrals (hmlint) per second", "value": leg["value"], "unit": "atoms/s",
           "n_gpus": 1, "steps": 20, "warmup": max(3, args.warmup), "ms_per_step": leg["ms"],
           "higher_is_better": True, "dtype": "f64", "data": "synthetic",
           "config": {"workload": "si_cube216" if args.workload == "cube216" else "si_cube8",
                      "natmtot": s.natmtot, "lmaxmat": s.basis.lmaxmat, "lmaxvr": leg["lmaxvr"],
                      "nrmt": leg["nrmt"]},
           "e2e": leg["e2e"], "roofline": leg["roofline"], "cpu_baseline": leg["cpu_baseline"],
           "gpu_launches": 2 * 20}
    print(json.dumps(out), flush=True)
    st.set_stream(None)
    st.close()
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--nk", type=int, default=27, help="k-points per step (profiling runs use fewer)")
    ap.add_argument("--skip-cpu", action="store_true", help="no CPU-baseline leg (profiling runs)")
    ap.add_argument("--skip-e2e", action="store_true", help="no host-pointer leg (profiling runs)")
    ap.add_argument("--skip-hmlint", action="store_true", help="no muffin-tin integral leg (profiling runs)")
    ap.add_argument("--skip-rttddft", action="store_true", help="no RT-TDDFT update leg (profiling runs)")
    ap.add_argument("--precision", default="ozaki_mod", choices=["fp64", "ozaki", "ozaki_mod"],
                    help="MT contraction arithmetic: ozaki_mod = int8 residues modulo coprime moduli, "
                         "ozaki = int8 slices (the native FP64 path is timed beside either)")
    ap.add_argument("--workload", default="cube216", choices=["cube8", "cube216", "cells256"],
                    help="cube216: 216-atom cell, one of its 4 k-points per step (the 8-atom batch runs as a "
                         "secondary leg); cube8: 8-atom cell, 27 k per step; cells256: 256 independent 2-atom "
                         "cells per step in one graph")
    ap.add_argument("--skip-adjoint", action="store_true", help="no adjoint leg")
    ap.add_argument("--kernel-config", type=int, default=-1,
                    help="split-precision kernel configuration (0..31); -1: the autotuner's choice (8-atom batch) "
                         "or the library default (216-atom cell)")
    ap.add_argument("--skip-eig", action="store_true", help="cube216: no eigenvalue comparison at Gamma")
    ap.add_argument("--dense-eig", action="store_true",
                    help="cube216: also compare the lowest 40 eigenvalues of two dense solves (about 4 minutes)")
    ap.add_argument("--skip-fp64", action="store_true", help="cube216: no FP64 leg and no accuracy comparison")
    ap.add_argument("--skip-cube8", action="store_true", help="cube216: no 8-atom secondary leg")
    ap.add_argument("--slices", type=int, default=7, help="int8 slices per operand (ozaki)")
    ap.add_argument("--moduli", type=int, default=0,
                    help="moduli of ozaki_mod (0: the fewest that keep 41 + log2(K)/2 bits per operand)")
    ap.add_argument("--leg", default="setup", choices=["setup", "hmlint"],
                    help="hmlint: only the muffin-tin integral generation of --workload (cube8 or cube216)")
    args = ap.parse_args()
    if args.impl == "reference":
        return run_reference(args)
    if args.leg == "hmlint":
        return run_hmlint(args)
    if args.workload == "cube216":
        return run_large(args)
    if args.workload == "cells256":
        return run_cells(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
