"""Benchmark: dsposv vs dposv time to an FP64 backward error at n = 32768.

One step = one plasma_dsposv solve (low-precision tile Cholesky + FP64
iterative refinement) of the mixed-precision configuration: n = 32768,
nrhs = 1, A = Q diag(lambda) Q^T with Q from Householder QR of an N(0,1)
matrix (seed 11), lambda log-spaced from 1 to 1/kappa, b = A x_true.  The
operands are resident in HBM (8.6 GB, larger than L2) and are passed to the
LAPACK-layout C entry point as device pointers.  Beside it the plain FP64
plasma_dposv is timed on the same matrix; the ratio is the speed-up.

value      : FP64-equivalent GFLOP/s of dsposv, (n^3/3 + 2 n^2 nrhs) / t.
e2e        : the same, through plasma_dsposv with HOST buffers (H2D of A and
             b and D2H of x inside the timed region).
roofline   : the dominant kernel (trailing update) of the timed region, timed
             by the library's own CUDA events on its launch stream.
cpu_baseline / --impl reference : the reference PLASMA itself, built from
             its sources into oracle/_ref (oracle/build_ref.sh) with
             OpenBLAS 0.3.15 single-threaded and its OpenMP tasks on all host
             cores, on the same n = 32768 system: one solve for
             cpu_baseline, one solve per step for the reference arm, which
             prints the same metric on the same workload.
Multi-GPU: the path does not shard (one matrix per GPU); N GPUs run N
independent replicas, timed as the max over ranks.
"""
import argparse
import ctypes
import json
import os
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "tests", "golden"))


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=3)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--n", type=int, default=32768)
    p.add_argument("--nrhs", type=int, default=1)
    p.add_argument("--kappa", type=float, default=1e5)
    p.add_argument("--mode", default="fp32", choices=["fp32", "tf32", "bf16", "auto"])
    p.add_argument("--refine", default="ir", choices=["ir", "gmres", "auto"])
    p.add_argument("--nb", type=int, default=0, help="0 = autotuned table")
    p.add_argument("--no-e2e", action="store_true")
    p.add_argument("--no-cpu", action="store_true")
    p.add_argument("--no-dposv", action="store_true")
    p.add_argument("--band-nb", default="0",
                   help="band workload: comma-separated tile sizes (0 = tuned)")
    p.add_argument("--band-kd", default="256,1024,4096",
                   help="band workload: comma-separated bandwidths")
    p.add_argument("--batch-count", type=int, default=4096,
                   help="matrices of the batched workload")
    p.add_argument("--kappas", default="1e2,1e5,1e8",
                   help="mixed workload: condition numbers")
    p.add_argument("--ns", default="8192,16384,32768", help="dposv workload: sizes")
    p.add_argument("--nbs", default="128,256,384,512", help="dposv workload: tile sizes")
    p.add_argument("--workload", default="dsposv",
                   choices=["dsposv", "mixed", "dposv", "adjoint", "batched", "inverse",
                            "band", "lu"],
                   help="dsposv: the headline; adjoint / batched: the differentiation "
                        "and batched-solve configurations, one JSON line each")
    return p.parse_args()


# the benchmark's metric, printed verbatim by both arms
METRIC = ("dsposv vs dposv time-to-FP64-backward-err at n=32768 on 1 B200; "
          "GFLOP/s, % roofline")
MODES = {"fp32": 0, "tf32": 1, "bf16": 2, "auto": 3}
UPDATE_DRAM_BYTES_PER_TILE = {"fp32": 384465}
REFINE = {"ir": 0, "gmres": 1, "auto": 2}


def dist_info():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def workload_config(args, nb):
    return {"workload": f"dsposv n={args.n} nrhs={args.nrhs} A=Q diag(lambda) Q^T "
                        f"kappa={args.kappa:g} seed 11, b = A x_true (seed 12), uplo=L",
            "factor": args.mode, "refinement": args.refine, "nb": nb,
            "l2": f"inputs larger than L2 (A is {args.n * args.n * 8 / 1e9:.1f} GB)"
                  if args.n * args.n * 8 > 126e6 else "A smaller than L2",
            "parallelism": "replicas x1"}


def flops_of(n, nrhs):
    return n ** 3 / 3.0 + 2.0 * n * n * nrhs


def make_system(n, nrhs, kappa, device, seed=11):
    """A = Q diag(lambda) Q^T (symmetric: row-major == column-major), b = A x."""
    import torch
    g = torch.Generator(device=device).manual_seed(seed)
    G = torch.randn(n, n, generator=g, device=device, dtype=torch.float64)
    Q, _ = torch.linalg.qr(G)
    del G
    lam = torch.logspace(0.0, -float(np.log10(kappa)), n, device=device,
                         dtype=torch.float64)
    A = (Q * lam) @ Q.T
    del Q
    A = 0.5 * (A + A.T)
    g2 = torch.Generator(device=device).manual_seed(seed + 1)
    xt = torch.randn(nrhs, n, generator=g2, device=device, dtype=torch.float64)
    B = (A @ xt.T).T.contiguous()          # nrhs x n row-major = n x nrhs col-major
    if A.is_cuda:
        torch.cuda.synchronize()
    return A.contiguous(), B, xt


def measured_peaks(torch):
    """Roofline denominators in TFLOP/s (hbm_gbs in GB/s).  BF16 and HBM from
    MEASURED_PEAKS.json; the FP64 and FP32/TF32 peaks are not in that file, so
    they are measured here the same way (cuBLAS GEMM, best of 5, CUDA
    events)."""
    peaks = {}
    try:
        mp = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
        peaks["bf16"] = mp.get("bf16_tflops")  # already TFLOP/s
        peaks["bf16_sustained"] = mp.get("bf16_tflops_sustained")
        peaks["hbm_gbs"] = mp.get("hbm_gbs")
        peaks["source"] = "MEASURED_PEAKS.json"
    except Exception:
        peaks.update({"bf16": 1590.0, "hbm_gbs": 6650.0, "source": "fallback"})

    def gemm_tf(dtype, tf32, n=8192, reps=5):
        torch.backends.cuda.matmul.allow_tf32 = tf32
        a = torch.randn(n, n, device="cuda", dtype=dtype)
        b = torch.randn(n, n, device="cuda", dtype=dtype)
        for _ in range(2):
            a @ b
        torch.cuda.synchronize()
        best = 1e9
        for _ in range(reps):
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record()
            a @ b
            e1.record()
            torch.cuda.synchronize()
            best = min(best, e0.elapsed_time(e1))
        torch.backends.cuda.matmul.allow_tf32 = False
        return 2.0 * n ** 3 / best / 1e9     # flops per ms / 1e9 = TFLOP/s

    peaks["fp64"] = gemm_tf(torch.float64, False)
    peaks["fp32"] = gemm_tf(torch.float32, False)
    peaks["tf32"] = gemm_tf(torch.float32, True)
    return peaks


class Clocks:
    """nvidia-smi sampling during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.p = None

    def start(self):
        try:
            self.p = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.p = None

    def stop(self):
        if self.p is None:
            return None
        time.sleep(0.25)
        self.p.terminate()
        try:
            out, _ = self.p.communicate(timeout=5)
        except Exception:
            self.p.kill()
            return None
        mhz, maxmhz, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in out.strip().splitlines():
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                mhz.append(float(f[1]))
                maxmhz = float(f[2])
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        if not mhz:
            return None
        return {"sm_mhz": float(np.median(mhz)), "sm_max_mhz": maxmhz,
                "reasons": sorted(reasons), "samples": len(mhz)}


def cpu_model():
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def host_system(A, B):
    """Column-major host copies of the device system (A symmetric, so its
    row-major bytes are its column-major ones; B is nrhs x n row-major)."""
    a = np.asfortranarray(A.cpu().numpy())
    b = np.asfortranarray(B.cpu().numpy().T)
    return a, b


def reference_dsposv(a, b, nb, threads):
    """One plasma_dsposv of the reference PLASMA itself (oracle/_ref: its own
    sources, OpenBLAS 0.3.15 single-threaded, OpenMP tasks on `threads`
    host cores) on host arrays; returns (seconds, info, iter)."""
    from oracle import ref
    ref.set_threads(threads)
    x = np.zeros_like(b, order="F")
    t0 = time.perf_counter()
    info, it = ref.dsposv(ref.LOWER, a, b, x, nb)
    return time.perf_counter() - t0, info, it


def cpu_baseline(a, b, nb=256):
    """The reference PLASMA on the host cores on one solve of the same
    workload (the bounded sample: one dsposv of the benchmark's own system)."""
    threads = os.cpu_count() or 1
    n, nrhs = b.shape
    dt, info, it = reference_dsposv(a, b, nb, threads)
    return {"value": flops_of(n, nrhs) / dt / 1e9, "unit": "GFLOP/s",
            "cores": threads, "kind": "reference",
            "sample": f"reference PLASMA plasma_dsposv (oracle/_ref, OpenBLAS 0.3.15 "
                      f"single-threaded, {threads} OpenMP threads on {cpu_model()}), one solve "
                      f"of the same n={n} nrhs={nrhs} system, nb={nb}: {dt:.2f} s, "
                      f"iter {it}, info {info}",
            "seconds": dt}


def reference_built():
    from oracle import ref
    return os.path.exists(ref.LIB_PATH)


def reference_sample(routine, n, extra, nb, threads, dt, info, it=None):
    return {"value": dt * 1e3, "unit": "ms", "cores": threads, "kind": "reference",
            "sample": f"reference PLASMA plasma_{routine} (oracle/_ref, OpenBLAS 0.3.15 "
                      f"single-threaded, {threads} OpenMP threads on {cpu_model()}), one "
                      f"solve of the same n={n}{extra} system, nb={nb}: {dt:.2f} s, "
                      f"info {info}" + ("" if it is None else f", iter {it}")}


def reference_dsgesv_cpu(a, b, nb=256):
    """The reference's own plasma_dsgesv on the host cores (one solve of the
    workload's system, host copies a, b in Fortran order): the cpu_baseline
    entry of the LU workload."""
    from oracle import ref
    threads = os.cpu_count() or 1
    ref.set_threads(threads)
    x = np.zeros(b.shape, order="F")
    t0 = time.perf_counter()
    info, it, _ = ref.dsgesv(a, b, x, nb)
    dt = time.perf_counter() - t0
    return reference_sample("dsgesv", a.shape[0], "", nb, threads, dt, info, it)


def reference_dpbsv_cpu(ab, kd, b, nb=256):
    """The reference's own plasma_dpbsv (lower band storage ab, (kd+1) x n,
    Fortran order) on the host cores: the band workload's cpu_baseline."""
    from oracle import ref
    threads = os.cpu_count() or 1
    ref.set_threads(threads)
    ab, x = np.asfortranarray(ab.copy()), np.asfortranarray(b.copy())
    t0 = time.perf_counter()
    info = ref.dpbsv(ref.LOWER, ab, kd, x, nb)
    dt = time.perf_counter() - t0
    return reference_sample("dpbsv", ab.shape[1], f" kd={kd}", nb, threads, dt, info)


def max_over_ranks(ms, world, device):
    """The job's step time: the slowest replica's (MAX over the ranks of the
    initialised process group; every rank gets it)."""
    if world <= 1:
        return ms
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(ms)], device=device, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return t.item()


def run_reference(args):
    """The reference arm: the reference PLASMA's own plasma_dsposv (built
    from its sources into oracle/_ref) on the same n = 32768 system, all
    host cores, OpenBLAS single-threaded; one step = one solve.  The system
    is generated on the GPU (the same generator as the GPU arm) and copied
    to host memory before the timed steps."""
    rank, world, _ = dist_info()
    if rank != 0:
        return 0
    import torch
    n, nrhs, nb = args.n, args.nrhs, (args.nb or 256)
    dev = "cuda" if torch.cuda.is_available() else "cpu"
    A, B, xt = make_system(n, nrhs, args.kappa, dev)
    a, b = host_system(A, B)
    xt = xt.cpu().numpy().T
    del A, B
    if dev == "cuda":
        torch.cuda.empty_cache()
    threads = os.cpu_count() or 1
    # one untimed solve warms the host (each reference solve allocates and
    # first-touches its own tile copies, so more warm-up changes nothing);
    # a 20-second solve per step keeps the arm within minutes
    warm = min(args.warmup, 1)
    secs, infos, iters = [], [], []
    for i in range(warm + args.steps):
        dt, info, it = reference_dsposv(a, b, nb, threads)
        if i >= warm:
            secs.append(dt)
            infos.append(info)
            iters.append(it)
    ms = float(np.mean(secs)) * 1e3
    value = flops_of(n, nrhs) / (ms / 1e3) / 1e9
    line = {
        "impl": "reference",
        "metric": METRIC,
        "value": value, "unit": "GFLOP/s", "n_gpus": world, "steps": args.steps,
        "warmup": warm, "warmup_requested": args.warmup, "ms_per_step": ms,
        "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32+f64",
        "data": "synthetic",
        "config": workload_config(args, nb),
        "step_ms": [t * 1e3 for t in secs],
        "iter": iters[-1], "info": infos[-1],
        "cpu_baseline": {"value": value, "unit": "GFLOP/s", "cores": threads,
                         "kind": "reference",
                         "sample": f"reference PLASMA plasma_dsposv (oracle/_ref, OpenBLAS "
                                   f"0.3.15 single-threaded, {threads} OpenMP threads on "
                                   f"{cpu_model()}), {args.steps} solves of the n={n} "
                                   f"nrhs={nrhs} system, nb={nb}"},
        "e2e": {"value": value, "unit": "GFLOP/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def run_adjoint(args):
    """Forward (potrf + potrs) and backward (the two adjoints) of
    logdet(A) + trace(B^T A^-1 B) through plasma_b200.autograd, A = G G^T/n + I
    (G ~ N(0,1), seed 3), B ~ N(0,1), nrhs = 8, n in {4096, 8192}, FP64 and
    FP32.  Device memory: the most held at the phase boundaries (inputs,
    autograd state, the library's workspace, which it keeps between calls),
    above the level before the inputs were made."""
    import torch
    import plasma_b200 as pb
    import plasma_b200.autograd as ag
    L = pb.lib()
    assert L.plasma_init() == 0
    rows = []
    for n in (4096, 8192):
        for dt in (torch.float64, torch.float32):
            torch.cuda.synchronize()
            free_base, total = torch.cuda.mem_get_info()
            g = torch.Generator(device="cuda").manual_seed(3)
            G = torch.randn(n, n, generator=g, device="cuda", dtype=torch.float64)
            A0 = (G @ G.T / n + torch.eye(n, device="cuda", dtype=torch.float64)).to(dt)
            B0 = torch.randn(n, 8, generator=g, device="cuda", dtype=torch.float64).to(dt)
            del G
            fwd, bwd, peak = [], [], 0          # bytes above free_base
            for rep in range(args.warmup + args.steps):
                A = A0.clone().requires_grad_(True)
                B = B0.clone().requires_grad_(True)
                torch.cuda.synchronize()
                free0, total = torch.cuda.mem_get_info()
                e = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
                e[0].record()
                f = ag.gaussian_nll(A, B)
                e[1].record()
                torch.cuda.synchronize()
                free1, _ = torch.cuda.mem_get_info()
                f.backward()
                e[2].record()
                torch.cuda.synchronize()
                free2, _ = torch.cuda.mem_get_info()
                peak = max(peak, free_base - min(free0, free1, free2))
                if rep >= args.warmup:
                    fwd.append(e[0].elapsed_time(e[1]))
                    bwd.append(e[1].elapsed_time(e[2]))
                del A, B, f
            flops_f = n ** 3 / 3 + 2 * n * n * 8
            flops_b = 4 * n ** 3 / 3 + 6 * n * n * 8
            rows.append({"n": n, "dtype": "f64" if dt == torch.float64 else "f32",
                         "forward_ms": min(fwd), "backward_ms": min(bwd),
                         "forward_gflops": flops_f / min(fwd) / 1e6,
                         "backward_gflops": flops_b / min(bwd) / 1e6,
                         "device_memory_gb": peak / 1e9})
    print(json.dumps({"workload": "adjoint", "metric": "forward + backward time of "
                      "logdet(A) + tr(B^T A^-1 B)", "unit": "ms", "steps": args.steps,
                      "warmup": args.warmup, "nrhs": 8, "results": rows}), flush=True)
    L.plasma_finalize()
    return 0


def run_inverse(args):
    """plasma_dpoinv / plasma_spoinv (potrf + potri) on device-resident A,
    n in {8192, 16384}.  A = G G^T/n + I (G ~ N(0,1), seed 3).  GFLOP/s counts the reference's
    flops (potrf n^3/3, potri 2n^3/3: trtri + lauum); the library's potri
    does 2n^3 (the tile sweeps on the identity), reported as
    executed_tflops.  Error: ||A inv(A) - I||_max."""
    import torch
    import plasma_b200 as pb
    L = pb.lib()
    assert L.plasma_init() == 0
    rows = []
    for n in (8192, 16384):
        g = torch.Generator(device="cuda").manual_seed(3)
        G = torch.randn(n, n, generator=g, device="cuda", dtype=torch.float64)
        A0 = G @ G.T / n + torch.eye(n, device="cuda", dtype=torch.float64)
        del G
        for dt, fn in ((torch.float64, "d"), (torch.float32, "s")):
            A1 = A0.to(dt)
            times = []
            for rep in range(args.warmup + args.steps):
                A = A1.clone()
                e0 = torch.cuda.Event(enable_timing=True)
                e1 = torch.cuda.Event(enable_timing=True)
                torch.cuda.synchronize()
                e0.record()
                rc = getattr(L, f"plasma_{fn}poinv")(pb.PlasmaLower, n, A.data_ptr(), n)
                e1.record()
                torch.cuda.synchronize()
                assert rc == 0, rc
                if rep >= args.warmup:
                    times.append(e0.elapsed_time(e1))
            # A holds the column-major result, i.e. its transpose: the lower
            # triangle of the inverse is the tensor's upper triangle
            inv = torch.triu(A.double()) + torch.triu(A.double(), 1).T
            err = (A0 @ inv - torch.eye(n, device="cuda", dtype=torch.float64)).abs().max().item()
            ms = min(times)
            rows.append({"routine": f"{fn}poinv", "n": n, "ms": ms,
                         "gflops": n ** 3 / ms / 1e6,
                         "executed_tflops": (n ** 3 / 3 + 2 * n ** 3) / ms / 1e9,
                         "max_error_A_invA_minus_I": err})
            del A, A1, inv
    print(json.dumps({"workload": "inverse", "metric": "time of the SPD inverse "
                      "(poinv = potrf + potri), device-resident A, uplo = L",
                      "unit": "ms", "steps": args.steps, "warmup": args.warmup,
                      "results": rows}), flush=True)
    L.plasma_finalize()
    return 0


def run_band(args):
    """plasma_dpbsv / plasma_spbsv (band Cholesky + the two band sweeps) on a
    device-resident SPD band matrix in LAPACK band storage, n = 32768 and
    kd in {256, 1024, 4096}, one right-hand side.  AB = U[-0.5, 0.5] with
    2 kd + 1 added to the diagonal (diagonally dominant), b ~ U[-1, 1]
    (seed 9).  GFLOP/s counts LAPACK's flops for dpbtrf (n (kd^2 + 3 kd))
    and dpbtrs (4 n kd nrhs); the error is the reference tester's residual
    ||b - A x||_inf / (n ||A||_F ||x||_inf).  cpu_baseline (first FP64 row
    per kd): the reference's own plasma_dpbsv (oracle/_ref) on the host
    cores, one solve of the same system, when that library is built."""
    import torch
    import plasma_b200 as pb
    L = pb.lib()
    assert L.plasma_init() == 0
    n, rows, ref_done = 32768, [], set()
    for kd in [int(v) for v in args.band_kd.split(",")]:
        g = torch.Generator(device="cuda").manual_seed(9)
        # column-major (kd+1) x n storage = row-major n x (kd+1)
        AB0 = torch.rand(n, kd + 1, generator=g, device="cuda", dtype=torch.float64) - 0.5
        AB0[:, 0] += 2 * kd + 1
        # entry (d, j) of the band storage is A(j+d, j): zero past the matrix
        corner = (torch.arange(n, device="cuda")[:, None]
                  + torch.arange(kd + 1, device="cuda")[None, :]) >= n
        AB0[corner] = 0.0
        b0 = torch.rand(n, generator=g, device="cuda", dtype=torch.float64) * 2 - 1
        for dt, fn, nb in [(dt, fn, int(v)) for dt, fn in ((torch.float64, "d"),
                                                          (torch.float32, "s"))
                           for v in args.band_nb.split(",")]:
            if nb > 0:
                L.plasma_set(pb.PlasmaTuning, pb.PlasmaDisabled)
                L.plasma_set(pb.PlasmaNb, nb)
            else:
                L.plasma_set(pb.PlasmaTuning, pb.PlasmaEnabled)
            AB1, b1 = AB0.to(dt), b0.to(dt)
            times, trf = [], []
            for rep in range(args.warmup + args.steps):
                for factor_only in (False, True):
                    AB, x = AB1.clone(), b1.clone()
                    e0 = torch.cuda.Event(enable_timing=True)
                    e1 = torch.cuda.Event(enable_timing=True)
                    torch.cuda.synchronize()
                    e0.record()
                    if factor_only:
                        rc = getattr(L, f"plasma_{fn}pbtrf")(pb.PlasmaLower, n, kd,
                                                             AB.data_ptr(), kd + 1)
                    else:
                        rc = getattr(L, f"plasma_{fn}pbsv")(pb.PlasmaLower, n, kd, 1,
                                                            AB.data_ptr(), kd + 1,
                                                            x.data_ptr(), n)
                    e1.record()
                    torch.cuda.synchronize()
                    assert rc == 0, rc
                    if rep >= args.warmup:
                        (trf if factor_only else times).append(e0.elapsed_time(e1))
            AB, x = AB1.clone(), b1.clone()
            assert getattr(L, f"plasma_{fn}pbsv")(pb.PlasmaLower, n, kd, 1, AB.data_ptr(),
                                                  kd + 1, x.data_ptr(), n) == 0
            nb_used = ctypes.c_int()
            L.plasma_get(pb.PlasmaNb, ctypes.byref(nb_used))
            xd = x.double()
            ax = AB0[:, 0] * xd
            for d in range(1, kd + 1):
                ax[d:] += AB0[:n - d, d] * xd[:n - d]
                ax[:n - d] += AB0[:n - d, d] * xd[d:]
            anorm = torch.sqrt((AB0[:, 0] ** 2).sum() + 2 * (AB0[:, 1:] ** 2).sum())
            res = ((b0 - ax).abs().max() / (n * anorm * xd.abs().max())).item()
            ms = min(times)
            flops = n * (kd * kd + 3.0 * kd) + 4.0 * n * kd
            row = {"routine": f"{fn}pbsv", "n": n, "kd": kd, "nb": nb_used.value,
                   "ms": ms, "pbtrf_ms": min(trf), "gflops": flops / ms / 1e6,
                   "tester_residual": res, "cpu_baseline": None}
            if fn == "d" and reference_built() and kd not in ref_done:
                # column-major (kd+1) x n band storage = AB0 (row-major n x (kd+1))
                ab_host = np.asfortranarray(AB0.cpu().numpy().T)
                b_host = np.asfortranarray(b0.cpu().numpy().reshape(n, 1))
                row["cpu_baseline"] = reference_dpbsv_cpu(ab_host, kd, b_host)
                ref_done.add(kd)
                del ab_host
            rows.append(row)
            del AB, AB1, x
    print(json.dumps({"workload": "band", "metric": "time of the SPD band solve "
                      "(pbsv = pbtrf + pbtrs), device-resident AB, uplo = L, nrhs = 1",
                      "unit": "ms", "steps": args.steps, "warmup": args.warmup,
                      "results": rows}), flush=True)
    L.plasma_finalize()
    return 0


def run_lu(args):
    """plasma_dsgesv (FP32 LU with partial pivoting + FP64 refinement) on a
    device-resident general A = U[-0.5, 0.5] (seed 9), n = 4096, one
    right-hand side b ~ U[-1, 1].  GFLOP/s counts LAPACK's dgetrf + dgetrs
    flops (2n^3/3 + 2n^2); the error is the reference tester's residual
    ||b - A x||_inf / (n ||A||_inf ||x||_inf).  cpu_baseline: the
    reference's own plasma_dsgesv (oracle/_ref) on the host cores, one solve
    of the same system, when that library is built."""
    import torch
    import plasma_b200 as pb
    L = pb.lib()
    assert L.plasma_init() == 0
    if args.nb:
        L.plasma_set(pb.PlasmaTuning, pb.PlasmaDisabled)
        L.plasma_set(pb.PlasmaNb, args.nb)
    rows = []
    for n in (4096,):
        g = torch.Generator(device="cuda").manual_seed(9)
        A = torch.rand(n, n, generator=g, device="cuda", dtype=torch.float64) - 0.5
        b = torch.rand(n, generator=g, device="cuda", dtype=torch.float64) * 2 - 1
        x = torch.zeros(n, device="cuda", dtype=torch.float64)
        piv = np.zeros(n, dtype=np.int32)
        it = ctypes.c_int()
        times = []
        for rep in range(args.warmup + args.steps):
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize()
            e0.record()
            rc = L.plasma_dsgesv(n, 1, A.data_ptr(), n, piv.ctypes.data, b.data_ptr(), n,
                                 x.data_ptr(), n, ctypes.byref(it))
            e1.record()
            torch.cuda.synchronize()
            assert rc == 0, rc
            if rep >= args.warmup:
                times.append(e0.elapsed_time(e1))
        # A holds the transpose of the column-major matrix: A_cm = A.T
        r = b - A.T @ x
        res = (r.abs().max() / (n * A.abs().sum(dim=0).max() * x.abs().max())).item()
        ms = min(times)
        row = {"routine": "dsgesv", "n": n, "ms": ms, "iter": it.value,
               "gflops": (2 * n ** 3 / 3 + 2 * n ** 2) / ms / 1e6,
               "tester_residual": res, "cpu_baseline": None}
        if reference_built():
            # the column-major matrix the library read is A.T
            a_host = np.asfortranarray(A.T.cpu().numpy())
            b_host = np.asfortranarray(b.cpu().numpy().reshape(n, 1))
            row["cpu_baseline"] = reference_dsgesv_cpu(a_host, b_host)
        rows.append(row)
    print(json.dumps({"workload": "lu", "metric": "time of the LU-based mixed-precision "
                      "solve (dsgesv), device-resident A, nrhs = 1",
                      "unit": "ms", "steps": args.steps, "warmup": args.warmup,
                      "results": rows}), flush=True)
    L.plasma_finalize()
    return 0


def run_batched(args):
    """4096 SPD systems, n uniform in [16, 512] (seed 5), A = G G^T / n + 0.1 I,
    b ~ N(0,1), FP64 and FP32: one batched posv (factor + solve) launch per
    step and the batched adjoints (potrs then potrf) of logdet(A) + b^T A^-1 b;
    systems/s and p50/p99 per-batch latency (CUDA events, one event pair per
    batch, CUDA-graph replay).  Beside it the plain path, plasma_dposv per
    matrix on device pointers, on the first 256 matrices (scaled to the
    batch)."""
    import torch
    import plasma_b200 as pb
    from plasma_b200.batched import Batch
    L = pb.lib()
    assert L.plasma_init() == 0
    rng = np.random.default_rng(5)
    sizes = rng.integers(16, 513, args.batch_count)
    out = {"workload": "batched", "metric": "batched SPD solves (uneven n in [16, 512])",
           "unit": "systems/s", "batch": len(sizes), "steps": args.steps,
           "warmup": args.warmup, "flops_per_batch": float(np.sum(sizes.astype(float) ** 3) / 3),
           "results": []}
    for dt in (torch.float64, torch.float32):
        b = Batch(sizes, dt, graph=True)
        g = torch.Generator(device="cuda").manual_seed(5)
        A0 = torch.zeros(b.matrix_elems, dtype=dt, device="cuda")
        B0 = torch.zeros(b.vector_elems, dtype=dt, device="cuda")
        for i, n in enumerate(sizes):
            n = int(n)
            G = torch.randn(n, n, generator=g, device="cuda", dtype=torch.float64)
            a = G @ G.T / n + 0.1 * torch.eye(n, device="cuda", dtype=torch.float64)
            A0[b.off_a[i]:b.off_a[i] + n * n] = a.reshape(-1).to(dt)
            B0[b.off_b[i]:b.off_b[i] + n] = torch.randn(n, generator=g, device="cuda",
                                                       dtype=torch.float64).to(dt)
        A, B, info = A0.clone(), B0.clone(), b.info_buffer()
        times, adj = [], []
        for rep in range(args.warmup + args.steps):
            A.copy_(A0)
            B.copy_(B0)
            e = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
            e[0].record()
            b.posv(A, B, info)
            e[1].record()
            Lbar = torch.zeros_like(A)
            Xbar = B0.clone()
            e[1].synchronize()
            e2 = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
            e2[0].record()
            b.potrs_adjoint(A, B, Xbar, Lbar)
            b.potrf_adjoint(A, Lbar)
            e2[1].record()
            torch.cuda.synchronize()
            if rep >= args.warmup:
                times.append(e[0].elapsed_time(e[1]))
                adj.append(e2[0].elapsed_time(e2[1]))
        assert not info.any()
        t = np.array(times)
        row = {"dtype": "f64" if dt == torch.float64 else "f32",
               "systems_per_s": len(sizes) / (np.median(t) / 1e3),
               "posv_ms_p50": float(np.percentile(t, 50)),
               "posv_ms_p99": float(np.percentile(t, 99)),
               "gflops": out["flops_per_batch"] / np.median(t) / 1e6,
               "adjoint_ms_p50": float(np.median(adj))}
        # the plain path, one matrix at a time (device pointers)
        nloop = min(256, len(sizes))
        f = L.plasma_dposv if dt == torch.float64 else L.plasma_sposv
        As = [A0[b.off_a[i]:b.off_a[i] + int(n) ** 2].clone() for i, n in enumerate(sizes[:nloop])]
        Bs = [B0[b.off_b[i]:b.off_b[i] + int(n)].clone() for i, n in enumerate(sizes[:nloop])]
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for i, n in enumerate(sizes[:nloop]):
            n = int(n)
            assert f(pb.PlasmaLower, n, 1, As[i].data_ptr(), n, Bs[i].data_ptr(), n) == 0
        torch.cuda.synchronize()
        loop_s = (time.perf_counter() - t0) * len(sizes) / nloop
        row["per_matrix_loop_ms"] = loop_s * 1e3
        row["speedup_vs_loop"] = loop_s * 1e3 / np.median(t)
        out["results"].append(row)
        b.close()
    print(json.dumps(out), flush=True)
    L.plasma_finalize()
    return 0


def _dsposv_cell(L, pb, A, B, X, xt, n, nrhs, mode, refine, steps, warmup):
    """One (factor precision, refinement) cell on a device-resident system:
    time of plasma_dsposv_ex (min over the timed solves, CUDA events), its
    report, the backward error ||b - A x||_inf / (||A||_inf ||x||_inf) and
    the forward error ||x - x_true||_inf / ||x_true||_inf."""
    import torch
    L.plasma_set(pb.PlasmaMixedPrecisionMode, MODES[mode])
    L.plasma_set(pb.PlasmaRefinement, REFINE[refine])
    it = ctypes.c_int()
    info = pb.plasma_dsposv_info_t()
    times, rc = [], 0
    for rep in range(warmup + steps):
        X.zero_()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record()
        rc = L.plasma_dsposv_ex(pb.PlasmaLower, n, nrhs, A.data_ptr(), n, B.data_ptr(), n,
                                X.data_ptr(), n, ctypes.byref(it), ctypes.byref(info))
        e1.record()
        torch.cuda.synchronize()
        if rep >= warmup:
            times.append(e0.elapsed_time(e1))
    row = {"factor": mode, "refinement": refine, "info": rc, "iter": it.value,
           "ms": min(times), "report": info.as_dict()}
    if rc == 0:
        Xc = X.T
        R = B.T - A @ Xc
        anorm = A.abs().sum(1).max().item()
        row["backward_error"] = (R.abs().max(0).values /
                                 (anorm * Xc.abs().max(0).values)).max().item()
        row["forward_error"] = ((Xc - xt.T).abs().max(0).values /
                                xt.T.abs().max(0).values).max().item()
    return row


def run_mixed(args):
    """The mixed-precision configuration in full: kappa in {1e2, 1e5, 1e8} x
    factor precision in {FP32 (three TF32 products), TF32, BF16}, each refined
    by IR for kappa <= 1e5 and by GMRES-IR for kappa = 1e8, at n = --n
    (32768), nrhs = 1, on device-resident operands.  Per cell: info, iter,
    the report of plasma_dsposv_ex (factor precision used, attempts, GMRES
    iterations, FP64 fallback), the time, the backward error and the forward
    error against x_true; per kappa the plain FP64 dposv time on the same
    matrix and its errors.  FP32 + IR is the reference's own configuration,
    with its failure semantics: where its FP32 factorisation breaks down the
    cell reports that info, as the reference does."""
    import torch
    import plasma_b200 as pb
    L = pb.lib()
    assert L.plasma_init() == 0
    if args.nb > 0:
        L.plasma_set(pb.PlasmaTuning, pb.PlasmaDisabled)
        L.plasma_set(pb.PlasmaNb, args.nb)
    n, nrhs = args.n, args.nrhs
    out = {"workload": "mixed", "metric": "dsposv time and accuracy per kappa and "
           "factor precision (vs plain FP64 dposv)", "n": n, "nrhs": nrhs, "unit": "ms",
           "steps": args.steps, "warmup": args.warmup,
           "backward_error_target": 50 * n * 2.0 ** -53, "results": []}
    kappas = [float(k) for k in args.kappas.split(",")]
    for kappa in kappas:
        A, B, xt = make_system(n, nrhs, kappa, "cuda")
        X = torch.zeros_like(B)
        # plain FP64 dposv on a copy (after one untimed call)
        Aw, Bw = A.clone(), B.clone()
        if kappa == kappas[0]:
            assert L.plasma_dposv(pb.PlasmaLower, n, nrhs, Aw.data_ptr(), n, Bw.data_ptr(),
                                  n) == 0
            Aw.copy_(A)
            Bw.copy_(B)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record()
        rc = L.plasma_dposv(pb.PlasmaLower, n, nrhs, Aw.data_ptr(), n, Bw.data_ptr(), n)
        e1.record()
        torch.cuda.synchronize()
        Xd = Bw.T
        anorm = A.abs().sum(1).max().item()
        dposv = {"info": rc, "ms": e0.elapsed_time(e1),
                 "backward_error": ((B.T - A @ Xd).abs().max(0).values /
                                    (anorm * Xd.abs().max(0).values)).max().item(),
                 "forward_error": ((Xd - xt.T).abs().max(0).values /
                                   xt.T.abs().max(0).values).max().item()}
        del Aw, Bw
        refine = "gmres" if kappa >= 1e8 else "ir"
        cells = []
        for mode in ("fp32", "tf32", "bf16"):
            cell = _dsposv_cell(L, pb, A, B, X, xt, n, nrhs, mode, refine, args.steps,
                                args.warmup)
            if cell["info"] == 0:
                cell["speedup_vs_dposv"] = dposv["ms"] / cell["ms"]
            cells.append(cell)
        if kappa >= 1e8:
            # the reference's own configuration on the same matrix
            cells.append(_dsposv_cell(L, pb, A, B, X, xt, n, nrhs, "fp32", "ir", 1, 0))
        out["results"].append({"kappa": kappa, "dposv": dposv, "cells": cells})
        del A, B, X, xt
        torch.cuda.empty_cache()
    L.plasma_set(pb.PlasmaMixedPrecisionMode, MODES["fp32"])
    L.plasma_set(pb.PlasmaRefinement, REFINE["ir"])
    print(json.dumps(out), flush=True)
    L.plasma_finalize()
    return 0


def make_diag_dominant(n, nrhs, seed, device):
    """A = sym(U[-0.5, 0.5]) + n I, B = U[-1, 1] (n x nrhs column-major, held
    as nrhs x n row-major), generated on the device."""
    import torch
    g = torch.Generator(device=device).manual_seed(seed)
    A = torch.rand(n, n, generator=g, device=device, dtype=torch.float64) - 0.5
    A = torch.tril(A) + torch.tril(A, -1).T
    A.diagonal().add_(n)
    B = torch.rand(nrhs, n, generator=g, device=device, dtype=torch.float64) * 2 - 1
    return A.contiguous(), B.contiguous()


def run_dposv(args):
    """Plain FP64 plasma_dposv (the FP64 tensor-core path), n in --ns
    (8192, 16384, 32768), nrhs = 16, A = sym(U[-0.5, 0.5]) + n I (seed 7),
    device-resident, lower storage; nb over {128, 256, 384, 512} and the
    library's tuned choice.  GFLOP/s = (n^3/3) / t (and the reference
    tester's flops, potrf + potrs), as a fraction of the FP64 tensor peak
    (cuBLAS DGEMM measured live).  --impl reference times the reference
    PLASMA's plasma_dposv (oracle/_ref) on the host cores instead."""
    import torch
    ns = [int(v) for v in args.ns.split(",")]
    nrhs = 16
    out = {"workload": "dposv", "metric": "plain FP64 dposv GFLOP/s (n^3/3 / t), "
           "fraction of FP64 tensor peak", "unit": "GFLOP/s", "nrhs": nrhs,
           "steps": args.steps, "warmup": args.warmup, "results": []}
    if args.impl == "reference":
        threads = os.cpu_count() or 1
        from oracle import ref
        ref.set_threads(threads)
        for n in ns:
            A, B = make_diag_dominant(n, nrhs, 7, "cuda" if torch.cuda.is_available() else "cpu")
            a, b = host_system(A, B)
            del A, B
            t = []
            for rep in range(max(1, args.steps)):
                x = b.copy(order="F")
                af = a.copy(order="F")
                t0 = time.perf_counter()
                info = ref.dposv(ref.LOWER, af, x, 256)
                t.append(time.perf_counter() - t0)
                assert info == 0, info
            ms = min(t) * 1e3
            out["results"].append({"n": n, "nb": 256, "ms": ms,
                                   "gflops": n ** 3 / 3 / ms / 1e6,
                                   "cores": threads, "cpu": cpu_model()})
        out["impl"] = "reference"
        print(json.dumps(out), flush=True)
        return 0
    import plasma_b200 as pb
    L = pb.lib()
    assert L.plasma_init() == 0
    peaks = measured_peaks(torch)
    out["fp64_peak_tflops"] = peaks["fp64"]
    for n in ns:
        A, B = make_diag_dominant(n, nrhs, 7, "cuda")
        Aw, Bw = torch.empty_like(A), torch.empty_like(B)
        rows = []
        for nb in [0] + [int(v) for v in args.nbs.split(",")]:
            if nb == 0:
                L.plasma_set(pb.PlasmaTuning, pb.PlasmaEnabled)
            else:
                L.plasma_set(pb.PlasmaTuning, pb.PlasmaDisabled)
                L.plasma_set(pb.PlasmaNb, nb)
            times = []
            for rep in range(args.warmup + args.steps):
                Aw.copy_(A)
                Bw.copy_(B)
                e0 = torch.cuda.Event(enable_timing=True)
                e1 = torch.cuda.Event(enable_timing=True)
                torch.cuda.synchronize()
                e0.record()
                rc = L.plasma_dposv(pb.PlasmaLower, n, nrhs, Aw.data_ptr(), n, Bw.data_ptr(), n)
                e1.record()
                torch.cuda.synchronize()
                assert rc == 0, rc
                if rep >= args.warmup:
                    times.append(e0.elapsed_time(e1))
            nbv = nb or L.plasma_tuning_get_potrf_nb(pb.PlasmaRealDouble, n)
            Xd = Bw.T
            R = B.T - A @ Xd
            anorm = A.abs().sum(1).max().item()
            res = (R.abs().max(0).values / (n * anorm * Xd.abs().max(0).values)).max().item()
            ms = min(times)
            rows.append({"nb": nbv, "tuned": nb == 0, "ms": ms,
                         "gflops": n ** 3 / 3 / ms / 1e6,
                         "tester_gflops": (n ** 3 / 3 + 2 * n * n * nrhs) / ms / 1e6,
                         "frac_fp64_peak": n ** 3 / 3 / ms / 1e9 / peaks["fp64"],
                         "tester_residual": res})
        best = min(rows, key=lambda r: r["ms"])
        # upper storage (factored through lower tiles) at the tuned nb
        L.plasma_set(pb.PlasmaTuning, pb.PlasmaEnabled)
        ut = []
        for rep in range(args.warmup + args.steps):
            Aw.copy_(A)
            Bw.copy_(B)
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize()
            e0.record()
            rc = L.plasma_dposv(pb.PlasmaUpper, n, nrhs, Aw.data_ptr(), n, Bw.data_ptr(), n)
            e1.record()
            torch.cuda.synchronize()
            assert rc == 0, rc
            if rep >= args.warmup:
                ut.append(e0.elapsed_time(e1))
        tuned = next(r for r in rows if r["tuned"])
        upper = {"ms": min(ut), "gflops": n ** 3 / 3 / min(ut) / 1e6,
                 "vs_lower_tuned": min(ut) / tuned["ms"]}
        out["results"].append({"n": n, "best": best, "upper": upper, "all": rows})
        del A, B, Aw, Bw
        torch.cuda.empty_cache()
    print(json.dumps(out), flush=True)
    L.plasma_finalize()
    return 0


def main():
    args = parse()
    if args.workload == "mixed":
        return run_mixed(args)
    if args.workload == "dposv":
        return run_dposv(args)
    if args.workload == "adjoint":
        return run_adjoint(args)
    if args.workload == "inverse":
        return run_inverse(args)
    if args.workload == "band":
        return run_band(args)
    if args.workload == "lu":
        return run_lu(args)
    if args.workload == "batched":
        return run_batched(args)
    if args.impl == "reference":
        return run_reference(args)

    import torch
    import plasma_b200 as pb

    rank, world, local = dist_info()
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))

    L = pb.lib()
    L.plasma_set(pb.PlasmaDevice, local)
    assert L.plasma_init() == 0
    if args.nb > 0:
        L.plasma_set(pb.PlasmaTuning, pb.PlasmaDisabled)
        L.plasma_set(pb.PlasmaNb, args.nb)
    L.plasma_set(pb.PlasmaMixedPrecisionMode, MODES[args.mode])
    L.plasma_set(pb.PlasmaRefinement, REFINE[args.refine])

    n, nrhs = args.n, args.nrhs
    peaks = measured_peaks(torch) if rank == 0 else {}
    A, B, xt = make_system(n, nrhs, args.kappa, "cuda")
    X = torch.zeros_like(B)
    it = ctypes.c_int()
    info = pb.plasma_dsposv_info_t()

    def dsposv():
        rc = L.plasma_dsposv_ex(pb.PlasmaLower, n, nrhs, A.data_ptr(), n, B.data_ptr(), n,
                                X.data_ptr(), n, ctypes.byref(it), ctypes.byref(info))
        assert rc == 0, rc

    def barrier():
        torch.cuda.synchronize()
        if world > 1:
            import torch.distributed as dist
            dist.barrier()

    for _ in range(args.warmup):
        dsposv()
    barrier()
    clocks = Clocks(local)
    clocks.start()
    pb.profile_enable(True)
    l0 = pb.launches()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    marks = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps + 1)]
    e0.record()
    marks[0].record()
    for i in range(args.steps):
        dsposv()
        marks[i + 1].record()
    e1.record()
    barrier()
    ms = e0.elapsed_time(e1) / args.steps
    step_ms = [marks[i].elapsed_time(marks[i + 1]) for i in range(args.steps)]
    launches = pb.launches() - l0
    prof = {k: pb.profile_query(k) for k in pb.KCLASS}
    pb.profile_enable(False)
    clk = clocks.stop()
    ms = max_over_ranks(ms, world, "cuda")

    # accuracy of the last solve
    Xc = X.T
    R = B.T - A @ Xc
    anorm = A.abs().sum(1).max().item()
    berr = (R.abs().max(0).values / (anorm * Xc.abs().max(0).values)).max().item()
    ferr = ((Xc - xt.T).abs().max(0).values / xt.T.abs().max(0).values).max().item()
    iters = it.value

    # plain FP64 dposv on the same matrix (A copied: dposv factors in place)
    dposv = None
    if not args.no_dposv and rank == 0:
        Aw = torch.empty_like(A)
        Bw = torch.empty_like(B)
        times = []
        for rep in range(2):
            Aw.copy_(A)
            Bw.copy_(B)
            torch.cuda.synchronize()
            f0 = torch.cuda.Event(enable_timing=True)
            f1 = torch.cuda.Event(enable_timing=True)
            pb.profile_enable(True)
            f0.record()
            rc = L.plasma_dposv(pb.PlasmaLower, n, nrhs, Aw.data_ptr(), n, Bw.data_ptr(), n)
            f1.record()
            torch.cuda.synchronize()
            assert rc == 0, rc
            if rep == 1:
                times.append(f0.elapsed_time(f1))
                dprof = pb.profile_query("update")
            pb.profile_enable(False)
        Xd = Bw.T
        Rd = B.T - A @ Xd
        berr_d = (Rd.abs().max(0).values / (anorm * Xd.abs().max(0).values)).max().item()
        dms = min(times)
        upd_tf = dprof["flops"] / dprof["ms"] / 1e9 if dprof["ms"] > 0 else None
        dposv = {"ms": dms, "gflops": flops_of(n, nrhs) / dms / 1e6,
                 "frac_fp64_peak": flops_of(n, nrhs) / dms / 1e9 / peaks["fp64"],
                 "update_kernel_tflops": upd_tf, "backward_error": berr_d}
        del Aw, Bw

    # end to end through host buffers: page-locked host copies of A and b,
    # the H2D upload of A's stored triangle and of b and the D2H of x inside
    # the timed region, through the LAPACK-layout entry point
    e2e = None
    if not args.no_e2e and rank == 0:
        ah = torch.empty_like(A, device="cpu").pin_memory()
        ah.copy_(A)                                   # symmetric: also column-major
        bh = torch.empty_like(B, device="cpu").pin_memory()
        bh.copy_(B)                                   # nrhs x n = column-major n x nrhs
        xh = torch.zeros_like(bh).pin_memory()
        L.plasma_dsposv_ex(pb.PlasmaLower, n, nrhs, ah.data_ptr(), n, bh.data_ptr(), n,
                           xh.data_ptr(), n, ctypes.byref(it), None)
        torch.cuda.synchronize()
        ets = []
        for _ in range(2):
            g0 = torch.cuda.Event(enable_timing=True)
            g1 = torch.cuda.Event(enable_timing=True)
            g0.record()
            rc = L.plasma_dsposv_ex(pb.PlasmaLower, n, nrhs, ah.data_ptr(), n, bh.data_ptr(),
                                    n, xh.data_ptr(), n, ctypes.byref(it), None)
            g1.record()
            torch.cuda.synchronize()
            assert rc == 0
            ets.append(g0.elapsed_time(g1))
        ems = min(ets)
        nbv = L.plasma_tuning_get_potrf_nb(pb.PlasmaRealFloat, n) if args.nb == 0 else args.nb
        h2d = sum((n - c0) * min(nbv, n - c0) for c0 in range(0, n, nbv)) * 8 + n * nrhs * 8
        e2e = {"value": flops_of(n, nrhs) / ems / 1e6, "unit": "GFLOP/s",
               "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(n * nrhs * 8),
               "ms_per_step": ems, "host_memory": "page-locked"}
        del ah, bh, xh
        # the same call on pageable host buffers (what a C caller passing
        # malloc'd arrays gets)
        ap = A.cpu()
        bp = B.cpu()
        xp = torch.zeros_like(bp)
        pts = []
        for _ in range(2):
            g0 = torch.cuda.Event(enable_timing=True)
            g1 = torch.cuda.Event(enable_timing=True)
            g0.record()
            rc = L.plasma_dsposv_ex(pb.PlasmaLower, n, nrhs, ap.data_ptr(), n, bp.data_ptr(),
                                    n, xp.data_ptr(), n, ctypes.byref(it), None)
            g1.record()
            torch.cuda.synchronize()
            assert rc == 0
            pts.append(g0.elapsed_time(g1))
        e2e["pageable"] = {"value": flops_of(n, nrhs) / min(pts) / 1e6,
                           "ms_per_step": min(pts), "host_memory": "pageable"}
        del ap, bp, xp

    cpu = None
    if not args.no_cpu and rank == 0:
        a_h, b_h = host_system(A, B)
        cpu = cpu_baseline(a_h, b_h, args.nb or 256)
        cpu.pop("seconds", None)
        del a_h, b_h

    if rank != 0:
        L.plasma_finalize()
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()
        return 0

    upd = prof["update"]
    # all factor modes run the trailing update on the tcgen05 tensor cores;
    # fp32 forms every FP32 product as three TF32 products (lo*hi + hi*lo +
    # hi*hi), so its tensor work is three times the algorithmic flops
    mode_peak = {"fp32": ("tf32", peaks.get("tf32"), 3), "tf32": ("tf32", peaks.get("tf32"), 1),
                 "bf16": ("bf16", peaks.get("bf16"), 1), "auto": ("bf16", peaks.get("bf16"), 1)}
    pk_name, pk, passes = mode_peak[args.mode]
    achieved = passes * upd["flops"] / upd["ms"] / 1e9 if upd["ms"] > 0 else None
    # DRAM bytes per 256 x 256 tile-update of the CTA-pair update kernel, read
    # + write, from one ncu capture (profiles/k_update_pair_tf32x3_n8192.md: a
    # bulk launch of 325 tile-updates); a launch's traffic grows with the
    # tiles it updates
    # (the algorithmic C read + write is 524288 bytes per tile-update)
    traffic = None
    dram_per_tile = UPDATE_DRAM_BYTES_PER_TILE.get(args.mode)
    nbv = args.nb or L.plasma_tuning_get_potrf_nb(pb.PlasmaRealFloat, n)
    if dram_per_tile and nbv == 256 and upd["launches"] > 0:
        tiles = upd["bytes"] / (8.0 * nbv * nbv)           # FP32 C read + write
        traffic = dram_per_tile * tiles / upd["launches"]
    value = world * flops_of(n, nrhs) / ms / 1e6
    line = {
        "metric": METRIC,
        "value": value, "unit": "GFLOP/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32+f64",
        "data": "synthetic",
        "config": dict(workload_config(args, nbv), parallelism=f"replicas x{world}"),
        "step_ms": step_ms,
        "iter": iters, "backward_error": berr, "forward_error": ferr,
        "backward_error_target": 50 * n * 2.0 ** -53,
        "dposv": dposv,
        "speedup_vs_dposv": (dposv["ms"] / ms) if dposv else None,
        "roofline": {"bound": "tensor",
                     "kernel": "k_update_pair trailing update (SYRK+GEMM, "
                               "tcgen05 cta_group::2)",
                     "achieved": achieved, "peak": pk, "unit": "TFLOP/s",
                     "frac": (achieved / pk) if achieved and pk else None,
                     "tensor_products_per_flop": passes,
                     "achieved_algorithmic": (achieved / passes) if achieved else None,
                     "peak_source": f"{pk_name} cuBLAS GEMM measured live (of measured)"
                     if pk_name != "bf16" else "MEASURED_PEAKS.json bf16_tflops (of measured)",
                     "traffic": traffic, "traffic_unit": "bytes per launch",
                     "launches": upd["launches"],
                     "avg_launch_ms": upd["ms"] / max(1, upd["launches"])},
        "phases_ms_per_step": {k: v["ms"] / args.steps for k, v in prof.items()},
        "peaks_tflops": peaks,
        "e2e": e2e,
        "cpu_baseline": cpu,
        "clocks": clk,
        "gpu_launches": int(launches),
    }
    print(json.dumps(line), flush=True)
    L.plasma_finalize()
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
