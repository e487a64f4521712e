"""Benchmark: batched symmetric eigendecompositions per second on B200.

Default workload: the ensemble-covariance-like (LETKF-style) batch,
L = 4096 matrices of n = 128, FP64, A = (k-1) I + Y^T Y with Y k x n iid
N(0,1)/sqrt(n), k = n; full eigenvalues + eigenvectors, sorted.  A step is
one solve of one batch; each step solves its own pristine copy (all copies
are resident in HBM before the timed region while they fit in half of the
free device memory, else a ring refilled inside the timed region; one batch
is 537 MB, larger than L2, so no flush is needed).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Under torchrun every rank solves its own batch (independent matrices, no
collective on the data path: weak scaling); time = max over ranks.

`--impl reference` times the reference method on the host cores instead:
the CPU restatement of the reference's tred1 -> tql2 -> hhtr2sy path
(oracle/, OpenMP over matrices, all threads), on a bounded sample per step.
"""
import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "eigeng-batched_b200"))


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=30)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference", "cusolver"])
    ap.add_argument("--n", type=int, default=128)
    ap.add_argument("--L", type=int, default=4096)
    ap.add_argument("--dtype", default="f64", choices=["f64", "f32"])
    ap.add_argument("--family", default="letkf", choices=["letkf", "symu", "clustered"])
    ap.add_argument("--method", default="tql2", choices=["tql2", "imtql2", "jacobi"])
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-extra", action="store_true",
                    help="skip the n=32 (L=16384) and n=256 (L=2048) FP64 figures added to the line")
    ap.add_argument("--uneven", type=int, default=0,
                    help="mixed-size workload: this many matrices, n uniform in [8, 512], A = Q diag(l) Q^T")
    ap.add_argument("--no-chosen", action="store_true",
                    help="skip the refined (tensor-core) form against the plain form at n=32/128/256")
    ap.add_argument("--no-learned", action="store_true", help="skip the learned warm start on the C5 family")
    ap.add_argument("--learned-epochs", type=int, default=10)
    ap.add_argument("--form", default="plain", choices=["plain", "refined", "learned"],
                    help="the solver form timed: the plain solve (default), the refined FP32->FP64 form on "
                         "--family/--n/--L, or the learned warm start on the theta family (--L matrices, n = 64)")
    ap.add_argument("--out", default=None, help="also append the JSON line to this file")
    return ap.parse_args()


def peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """Samples nvidia-smi clocks and throttle reasons around the timed
    region.  Started before the warm-up (nvidia-smi takes a moment to print
    its first sample), every sample is timestamped, and summary() keeps the
    samples inside the timed window; a window shorter than the sampling
    period keeps the nearest samples instead, taken under the same load."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    PERIOD_MS = 50

    def __init__(self, gpu):
        self.gpu = gpu
        self.proc = None
        self.lines = []  # (host time, csv line)

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), "--query-gpu=" + self.Q,
                                          "--format=csv,noheader,nounits", "-lms", str(self.PERIOD_MS)],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
            t_end = time.perf_counter() + 5.0
            while not self.lines and time.perf_counter() < t_end and self.proc.poll() is None:
                time.sleep(0.01)
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append((time.perf_counter(), line.strip()))

    def stop(self):
        if self.proc is not None:
            time.sleep(2.0 * self.PERIOD_MS / 1000.0)  # the samples just after the window
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
            self.proc = None

    @staticmethod
    def _parse(ln):
        f = [x.strip() for x in ln.split(",")]
        if len(f) < 9:
            return None
        try:
            return float(f[1]), float(f[2]), f[5:9]
        except ValueError:
            return None

    def summary(self, w0=None, w1=None):
        rows = [(t, r) for t, r in ((t, self._parse(ln)) for t, ln in self.lines) if r is not None]
        if w0 is not None and w1 is not None and rows:
            inside = [(t, r) for t, r in rows if w0 <= t <= w1]
            if not inside:  # window shorter than the period: the nearest samples
                mid = 0.5 * (w0 + w1)
                inside = sorted(rows, key=lambda x: abs(x[0] - mid))[:2]
            rows = inside
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for _, (c, m, flags) in rows:
            sm.append(c)
            mx.append(m)
            for nm, v in zip(names, flags):
                if v.lower() == "active":
                    reasons.add(nm)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"], "samples": 0}
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": float(max(mx)), "reasons": sorted(reasons),
                "samples": len(sm)}


def make_batch(torch, family, L, n, dtype, seed, device):
    """Seeded synthetic batch generated on the device (column-major matrices,
    symmetric).  LETKF-style: (n-1) I + Y^T Y, Y n x n iid N(0,1)/sqrt(n)."""
    if family == "clustered":
        return make_family_batch(torch, family, L, n, seed, device).to(dtype)
    g = torch.Generator(device=device)
    g.manual_seed(seed)
    out = torch.empty((L, n, n), dtype=dtype, device=device)
    step = 256
    for s in range(0, L, step):
        e = min(L, s + step)
        if family == "letkf":
            y = torch.randn((e - s, n, n), generator=g, dtype=torch.float64, device=device) / np.sqrt(n)
            a = y.transpose(1, 2) @ y + (n - 1) * torch.eye(n, dtype=torch.float64, device=device)
        else:
            b = torch.rand((e - s, n, n), generator=g, dtype=torch.float64, device=device) * 2 - 1
            a = 0.5 * (b + b.transpose(1, 2))
        out[s:e] = a.to(dtype)
    return out


FAMILY_TEXT = {
    "letkf": "LETKF-like (n-1) I + Y^T Y, Y iid N(0,1)/sqrt(n)",
    "symu": "(B + B^T)/2, B iid U[-1,1]",
    "clustered": "Q diag(l) Q^T, l in clusters of eight values 1e-8 apart, 0.1 between clusters",
}


class FreshInputs:
    """A pristine copy of `base` for each solve (a solve overwrites its
    input).  All of them are made before the timed region when they fit in
    half of the free device memory; otherwise a ring of as many as fit is
    kept and a reused slot is refilled from `base` on the current stream
    just before its solve, inside the timed region (a conservative number:
    the refill's device copy is timed with the solve)."""

    def __init__(self, torch, base, count):
        free, _ = torch.cuda.mem_get_info(base.device)
        per = base.numel() * base.element_size()
        self.r = max(2, min(count, int(0.5 * free) // max(1, per)))
        self.base = base
        self.bufs = [base.clone() for _ in range(self.r)]
        self.used = 0

    def reset(self):
        """Refill every slot (outside a timed region) for another pass."""
        for b in self.bufs:
            b.copy_(self.base)
        self.used = 0

    def next(self):
        i = self.used
        self.used += 1
        b = self.bufs[i % self.r]
        if i >= self.r:
            b.copy_(self.base)
        return b

    def note(self):
        if self.used > self.r:
            return f"inputs larger than L2 (ring of {self.r} device copies, refilled from the original inside the timed region)"
        return "inputs larger than L2 (fresh copy per step)"


def measured_traffic(kernel, dtype, n):
    """DRAM bytes per matrix (read + write) of a phase kernel from the
    committed ncu summary profiles/dram_traffic.txt, or None."""
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "profiles", "dram_traffic.txt")
    if not os.path.exists(path):
        return None
    with open(path) as f:
        for ln in f:
            parts = ln.split()
            if len(parts) >= 4 and not ln.startswith("#") and parts[0] == kernel and parts[1] == dtype \
                    and parts[2] == str(n):
                return float(parts[3])
    return None


def alg_bytes(n, esize):
    """Compulsory bytes per matrix: read A, write V and w."""
    return esize * (2 * n * n + n)


def phase_bytes(n, esize, recs):
    """Algorithmic bytes per matrix of each phase: 1 reads A and writes Q, d, e;
    2 reads d, e and writes the rotation records and w; 3 reads Q, the
    records and w and writes V and w."""
    rb = 2 * esize * recs
    return (esize * (2 * n * n + 2 * n), esize * 3 * n + rb, esize * (2 * n * n + 2 * n) + rb)


def cpu_time_oracle(a_np, n, method, budget_s, nthreads):
    """Times the CPU restatement (the -O3 -march=native build of oracle/,
    compiled on this machine) on a bounded sample: re-solves fresh copies
    of the sample until budget_s seconds have passed (at least once)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    O.lib(fast=True)
    done, t0 = 0, time.perf_counter()
    while True:
        a = a_np.copy()
        O.eigen_batch(a, n, method=method, nthreads=nthreads, fast=True)
        done += a_np.shape[0]
        el = time.perf_counter() - t0
        if el >= budget_s:
            return done / el, done, el


CPU_SAMPLE = 1024  # matrices of the workload in a CPU sample


def workload_config(args, world, l2_note):
    """The config dict of a bench line; the reference arm reports the same."""
    return {"workload": f"{args.family} L={args.L} n={args.n} {args.dtype} {args.method} sorted",
            "L_per_gpu": args.L, "n": args.n, "l2_flush": l2_note,
            "parallelism": f"replicas x{world} (independent matrices)"}


def run_reference(args):
    """Reference arm: the reference method on the host cores -- the CPU
    restatement of its tred1 -> tql2 -> hhtr2sy path (the reference's own
    CPU path, Fortran EISPACK, is not in its tree), all host threads, on
    the first CPU_SAMPLE matrices of the same batch our arm solves (same
    generator and seed), a fresh copy per step."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    import torch
    nth = os.cpu_count() or 1
    dev = torch.device("cuda", 0) if torch.cuda.is_available() else torch.device("cpu")
    dt = torch.float64 if args.dtype == "f64" else torch.float32
    n = args.n
    sample = min(args.L, CPU_SAMPLE)
    a_np = make_batch(torch, args.family, sample, n, dt, seed=1234, device=dev).cpu().numpy()
    method = {"tql2": 0, "imtql2": 1, "jacobi": 2}[args.method]
    for _ in range(args.warmup):
        cpu_time_oracle(a_np, n, method, 0.0, nth)
    rates = []
    for _ in range(args.steps):
        r, cnt, el = cpu_time_oracle(a_np, n, method, 0.0, nth)
        rates.append(r)
    value = float(np.median(rates))
    line = {
        "impl": "reference", "metric": f"eigendecomps/s (n={n}, {args.dtype}, {args.family}, L={args.L})",
        "value": value, "unit": "matrices/s", "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1000.0 * args.L / value, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": args.dtype, "data": "synthetic, seeded on device: " + FAMILY_TEXT[args.family],
        # a fresh copy per step, like our arm; the 1024-matrix sample (134 MB
        # at n=128 FP64) is also larger than the host CPU's caches
        "config": workload_config(args, args.gpus, "inputs larger than L2 (fresh copy per step)"),
        "cpu_baseline": {"value": value, "unit": "matrices/s", "cores": nth, "kind": "port",
                         "sample": f"the first {sample} matrices of the workload batch, one fresh-copy solve per step "
                                   f"(median of {args.steps}); ms_per_step scales to L={args.L}"},
        "e2e": {"value": value, "unit": "matrices/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    if args.out:
        with open(args.out, "a") as f:
            f.write(json.dumps(line) + "\n")


def run_cusolver(args):
    """Reported baseline on the same GPU: cuSOLVER's batched dense
    eigensolver (cusolverDnXsyevBatched; for n <= 32 also syevjBatched with
    the reference's settings, tolerance 512 eps / 16 eps and 10 sweeps,
    cusolver.hpp:23-25,108-110), on the same device-resident inputs and
    timing rules as this library's arm (fresh copy per step, CUDA events)."""
    import ctypes
    import torch
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if rank != 0:
        return
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    # the cuSOLVER that ships with torch, consistent with the cuBLAS torch has
    # already loaded (the system one may need a newer cuBLAS)
    import nvidia.cusolver
    lib = ctypes.CDLL(os.path.join(list(nvidia.cusolver.__path__)[0], "lib", "libcusolver.so.11"))
    P, I, I64, SZ = ctypes.c_void_p, ctypes.c_int, ctypes.c_int64, ctypes.c_size_t
    dt = torch.float64 if args.dtype == "f64" else torch.float32
    cdt = 1 if dt == torch.float64 else 0  # CUDA_R_64F / CUDA_R_32F
    n, L = args.n, args.L
    h, prm = P(), P()
    assert lib.cusolverDnCreate(ctypes.byref(h)) == 0
    assert lib.cusolverDnCreateParams(ctypes.byref(prm)) == 0
    stream = torch.cuda.current_stream(dev)
    assert lib.cusolverDnSetStream(h, P(stream.cuda_stream)) == 0
    base = make_batch(torch, args.family, L, n, dt, seed=1234, device=dev)
    inp = FreshInputs(torch, base, args.steps + args.warmup)
    w = torch.empty((L, n), dtype=dt, device=dev)
    info = torch.zeros(L, dtype=torch.int32, device=dev)
    lib.cusolverDnXsyevBatched_bufferSize.argtypes = [P, P, I, I, I64, I, P, I64, I, P, I, ctypes.POINTER(SZ),
                                                      ctypes.POINTER(SZ), I64]
    lib.cusolverDnXsyevBatched.argtypes = [P, P, I, I, I64, I, P, I64, I, P, I, P, SZ, P, SZ, P, I64]
    dws, hws = SZ(0), SZ(0)
    st = lib.cusolverDnXsyevBatched_bufferSize(h, prm, 1, 1, n, cdt, P(base.data_ptr()), n, cdt, P(w.data_ptr()),
                                               cdt, ctypes.byref(dws), ctypes.byref(hws), L)
    if st != 0:
        print(json.dumps({"impl": "cusolver", "unavailable": f"cusolverDnXsyevBatched_bufferSize status {st}"}))
        return
    dbuf = torch.empty(max(dws.value, 16), dtype=torch.uint8, device=dev)
    hbuf = ctypes.create_string_buffer(max(hws.value, 16))

    def solve(a):
        return lib.cusolverDnXsyevBatched(h, prm, 1, 1, n, cdt, P(a.data_ptr()), n, cdt, P(w.data_ptr()), cdt,
                                          P(dbuf.data_ptr()), dws.value, hbuf, hws.value, P(info.data_ptr()), L)

    def timed(fn):
        inp.reset()
        for i in range(args.warmup):
            assert fn(inp.next()) == 0
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for i in range(args.steps):
            assert fn(inp.next()) == 0
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / args.steps

    ms = timed(solve)
    line = {
        "impl": "cusolver", "routine": "cusolverDnXsyevBatched",
        "metric": f"eigendecomps/s (n={n}, {args.dtype}, {args.family}, L={L})",
        "value": L / (ms / 1000.0), "unit": "matrices/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": args.dtype,
        "data": "synthetic, seeded on device: " + FAMILY_TEXT[args.family],
        "config": {"workload": f"{args.family} L={L} n={n} {args.dtype}", "L_per_gpu": L, "n": n},
        "info_nonzero": int((info != 0).sum().item()),
    }
    if n <= 32:
        sinfo = P()
        assert lib.cusolverDnCreateSyevjInfo(ctypes.byref(sinfo)) == 0
        lib.cusolverDnXsyevjSetTolerance.argtypes = [P, ctypes.c_double]
        lib.cusolverDnXsyevjSetMaxSweeps.argtypes = [P, I]
        lib.cusolverDnXsyevjSetTolerance(sinfo, 512 * 2.0 ** -52 if dt == torch.float64 else 16 * 2.0 ** -23)
        lib.cusolverDnXsyevjSetMaxSweeps(sinfo, 10)
        pre = "D" if dt == torch.float64 else "S"
        fb = getattr(lib, f"cusolverDn{pre}syevjBatched_bufferSize")
        fs = getattr(lib, f"cusolverDn{pre}syevjBatched")
        fb.argtypes = [P, I, I, I, P, I, P, ctypes.POINTER(I), P, I]
        fs.argtypes = [P, I, I, I, P, I, P, P, I, P, P, I]
        lw = I(0)
        assert fb(h, 1, 1, n, P(base.data_ptr()), n, P(w.data_ptr()), ctypes.byref(lw), sinfo, L) == 0
        work = torch.empty(max(lw.value, 1), dtype=dt, device=dev)
        msj = timed(lambda a: fs(h, 1, 1, n, P(a.data_ptr()), n, P(w.data_ptr()), P(work.data_ptr()), lw.value,
                                 P(info.data_ptr()), sinfo, L))
        line["syevjBatched"] = {"value": L / (msj / 1000.0), "unit": "matrices/s", "ms_per_step": msj,
                                "tolerance": "512 eps (FP64) / 16 eps (FP32)", "max_sweeps": 10}
        lib.cusolverDnDestroySyevjInfo(sinfo)
    print(json.dumps(line), flush=True)
    if args.out:
        with open(args.out, "a") as f:
            f.write(json.dumps(line) + "\n")
    lib.cusolverDnDestroyParams(prm)
    lib.cusolverDnDestroy(h)


def make_uneven(torch, L, dtype, seed, device):
    """Mixed-size batch: n_k iid uniform in [8, 512]; A_k = Q diag(l) Q^T with
    Q from the QR factorization of an iid N(0,1) matrix and l log-spaced
    from 1 to 1e6 with random signs.  Returns (flat A, orders)."""
    rng = np.random.default_rng(seed)
    ns = rng.integers(8, 513, size=L)
    g = torch.Generator(device=device)
    g.manual_seed(seed)
    parts = [None] * L
    for n in np.unique(ns):
        idx = np.nonzero(ns == n)[0]
        x = torch.randn((len(idx), n, n), generator=g, dtype=torch.float64, device=device)
        q, _ = torch.linalg.qr(x)
        lam = torch.logspace(0, 6, int(n), dtype=torch.float64, device=device)
        sgn = torch.where(torch.rand((len(idx), n), generator=g, device=device, dtype=torch.float64) < 0.5, -1.0, 1.0)
        a = (q * (lam * sgn)[:, None, :]) @ q.transpose(1, 2)
        a = 0.5 * (a + a.transpose(1, 2))
        for j, k in enumerate(idx):
            parts[k] = a[j].transpose(0, 1).reshape(-1)  # column-major
    return torch.cat(parts).to(dtype).contiguous(), [int(x) for x in ns]


def run_uneven_bench(args):
    """Mixed-size batch through eigen_GPU_batch_uneven_* (inputs resident,
    a fresh copy per step, CUDA events).  Under torchrun the batch is split
    across ranks by cost (n^3, longest-processing-time, eigeng_b200.multi
    .shard_uneven) and each rank solves its share: a fixed total batch
    (strong scaling), time = max over ranks, no collective on the data path.
    The line also times the reference's usage on the same matrices: one
    uniform call per distinct order, one after another on one stream."""
    import torch
    import torch.distributed as dist
    import eigeng_b200 as E
    from eigeng_b200.multi import shard_uneven
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", device_id=dev, timeout=datetime.timedelta(seconds=300))
    dt = torch.float64 if args.dtype == "f64" else torch.float32
    full, ns_all = make_uneven(torch, args.uneven, dt, 1234, dev)
    mine = shard_uneven(ns_all, world)[rank] if world > 1 else list(range(len(ns_all)))
    offs_all = np.concatenate([[0], np.cumsum(np.array(ns_all, dtype=np.int64) ** 2)])
    ns = [int(ns_all[k]) for k in mine]
    base = torch.cat([full[offs_all[k]:offs_all[k + 1]] for k in mine]).contiguous() if world > 1 else full
    del full

    def sync_max(v):
        if world > 1:
            t = torch.tensor([v], dtype=torch.float64, device=dev)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            return float(t.item())
        return v

    inp = FreshInputs(torch, base, args.steps + args.warmup)
    for i in range(args.warmup):
        E.solve_uneven(inp.next(), ns)
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for i in range(args.steps):
        w, info = E.solve_uneven(inp.next(), ns)
    e1.record()
    torch.cuda.synchronize()
    ms = sync_max(e0.elapsed_time(e1) / args.steps)
    info_bad = int((info != 0).sum().item())
    del inp
    # the reference's usage on such a batch: one uniform call per distinct
    # order, one after another on one stream (same matrices, packed by order)
    nsa = np.array(ns)
    offs = np.concatenate([[0], np.cumsum(nsa.astype(np.int64) ** 2)])
    groups = {int(n): np.nonzero(nsa == n)[0] for n in np.unique(nsa)}
    packed = {n: torch.stack([base[offs[k]:offs[k + 1]] for k in idx]).reshape(len(idx), n, n).contiguous()
              for n, idx in groups.items()}
    wks = {n: E.workspace(len(idx), n, n, dt, dev) for n, idx in groups.items()}
    wss = {n: torch.empty((len(idx), n), dtype=dt, device=dev) for n, idx in groups.items()}
    per_order = []
    for rep in range(args.warmup + min(args.steps, 3)):
        cps = {n: p_.clone() for n, p_ in packed.items()}
        torch.cuda.synchronize()
        g0, g1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        g0.record()
        for n in groups:
            E.eigen_GPU_batch_ex(cps[n], wss[n], wks[n], n)
        g1.record()
        torch.cuda.synchronize()
        if rep >= args.warmup:
            per_order.append(g0.elapsed_time(g1))
        del cps
    ms_po = sync_max(float(np.median(per_order)))
    line = {"metric": f"eigendecomps/s (uneven n~U[8,512], {args.dtype}, L={args.uneven})",
            "value": args.uneven / (ms / 1000.0), "unit": "matrices/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "strong",
            "vs_baseline": None, "dtype": args.dtype,
            "data": "synthetic, seeded: Q diag(l) Q^T, l log-spaced 1..1e6 with random signs",
            "config": {"workload": f"uneven L={args.uneven} n~U[8,512] {args.dtype} tql2 sorted",
                       "elements": int(offs_all[-1]), "distinct_n": len(set(ns_all)),
                       "parallelism": f"cost-balanced shards x{world}", "l2_flush": "inputs larger than L2"},
            "info_nonzero": info_bad,
            "per_order_calls": {"matrices_per_s": args.uneven / (ms_po / 1000.0), "ms": ms_po,
                                "what": "one eigen_GPU_batch_ex call per distinct order, one stream"}}
    if rank == 0:
        print(json.dumps(line), flush=True)
        if args.out:
            with open(args.out, "a") as f:
                f.write(json.dumps(line) + "\n")
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()

def make_family_batch(torch, family, L, n, seed, device):
    """FP64 batches of the metric's families on the device: 'symu' (B + B^T)/2
    with B iid U[-1, 1], 'letkf' (n-1) I + Y^T Y, and 'clustered': Q diag(l)
    Q^T with Q from the QR factorization of an iid N(0,1) matrix and l in
    clusters of eight values 1e-8 apart, 0.1 between clusters."""
    if family != "clustered":
        return make_batch(torch, family, L, n, torch.float64, seed, device)
    g = torch.Generator(device=device)
    g.manual_seed(seed)
    out = torch.empty((L, n, n), dtype=torch.float64, device=device)
    idx = torch.arange(n, device=device, dtype=torch.float64)
    lam = torch.floor(idx / 8) * 0.1 + torch.remainder(idx, 8) * 1e-8 + 1.0
    for s in range(0, L, 256):
        e = min(L, s + 256)
        q, r = torch.linalg.qr(torch.randn((e - s, n, n), generator=g, dtype=torch.float64, device=device))
        q = q * torch.sign(torch.diagonal(r, dim1=1, dim2=2))[:, None, :]
        a = (q * lam[None, None, :]) @ q.transpose(1, 2)
        out[s:e] = 0.5 * (a + a.transpose(1, 2))
    return out


def timed_solves(torch, base, steps, warmup, fn, stream):
    """Device time (ms per solve) of fn over fresh copies of base."""
    inp = FreshInputs(torch, base, steps + warmup)
    last = None
    for _ in range(warmup):
        last = inp.next()
        fn(last)
    torch.cuda.synchronize()
    t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    t0.record(stream)
    for _ in range(steps):
        fn(inp.next())
    t1.record(stream)
    torch.cuda.synchronize()
    return t0.elapsed_time(t1) / steps, last


def gate_in_packed_solve(torch, E, base, n, stream, steps):
    """The packed solve alone against the packed solve with the accuracy
    gate in the same call (eigen_GPU_batch_packed_check), same packed
    inputs, same timing rules; plus the gate's verdict."""
    L = base.shape[0]
    ap = E.pack_upper(base, n)
    dt = base.dtype
    wk = E.workspace(L, n, n, dt, base.device)
    z = torch.empty_like(base)
    w = torch.empty((L, n), dtype=dt, device=base.device)
    info = torch.zeros(L, dtype=torch.int32, device=base.device)
    import ctypes
    e1 = torch.empty(L, dtype=torch.float64, device=base.device)
    e2 = torch.empty(L, dtype=torch.float64, device=base.device)
    fl = torch.empty(L, dtype=torch.int32, device=base.device)
    o = E.Opts(0, 1, 100, 0, 0, 0)
    sfx = "DP" if dt == torch.float64 else "FP"
    plain = getattr(E.lib(), "eigen_GPU_batch_packed_" + sfx)
    checked = getattr(E.lib(), "eigen_GPU_batch_packed_check_" + sfx)
    st = E._stream(stream)

    def run(with_gate):
        if with_gate:
            return checked(L, n, E._ptr(ap), E._ptr(z), n, E._ptr(w), E._ptr(wk), wk.numel(), E._ptr(info),
                           ctypes.byref(o), E._ptr(e1), E._ptr(e2), E._ptr(fl), st)
        return plain(L, n, E._ptr(ap), E._ptr(z), n, E._ptr(w), E._ptr(wk), wk.numel(), E._ptr(info),
                     ctypes.byref(o), st)
    out = {}
    for name, g in (("packed_solve", False), ("packed_solve_with_gate", True)):
        for _ in range(3):
            assert run(g) == 0
        torch.cuda.synchronize()
        t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        t0.record(stream)
        for _ in range(steps):
            run(g)
        t1.record(stream)
        torch.cuda.synchronize()
        out[name] = {"ms": t0.elapsed_time(t1) / steps}
    out["overhead"] = out["packed_solve_with_gate"]["ms"] / out["packed_solve"]["ms"] - 1.0
    out["gate_flags"] = int((fl != 0).sum())
    out["max_err1"] = float(e1.max())
    out["max_err2"] = float(e2.max())
    return out


def chosen_vs_plain(torch, E, args, stream):
    """The metric's comparison at n = 32, 128, 256 (FP64): the plain form
    (tridiagonal + QL) against the refined form (FP32 solve, tensor-core
    Ogita-Aishima refinement to FP64), same inputs, same timing rules; each
    with the reference's gate (err1 residual, err2 orthogonality) on its
    last warm-up result.  'chosen' is the faster at equal gate outcome."""
    out = {}
    steps = max(3, min(args.steps, 10))
    for fam, n, L in (("symu", 32, 16384), ("letkf", 128, 4096), ("clustered", 256, 2048)):
        base = make_family_batch(torch, fam, L, n, 4242, torch.device("cuda", torch.cuda.current_device()))
        w = torch.empty((L, n), dtype=torch.float64, device=base.device)
        info = torch.zeros(L, dtype=torch.int32, device=base.device)
        wk = E.workspace(L, n, n, torch.float64, base.device)
        ms_p, lp = timed_solves(torch, base, steps, 3, lambda a: E.eigen_GPU_batch_ex(a, w, wk, n, info=info,
                                                                                      stream=stream), stream)
        e1, e2, fl = E.check(base, w, lp, n)
        plain = {"matrices_per_s": L / ms_p * 1e3, "ms": ms_p, "gate_flags": int((fl != 0).sum()),
                 "max_err1": float(e1.max()), "max_err2": float(e2.max())}
        del wk
        rwk = E.refine_workspace(L, n, n, device=base.device)
        holder = {}

        def refined(a):
            holder["w"], holder["info"], holder["it"] = E.solve_refined(a, n, wk=rwk, stream=stream)
        ms_r, lr = timed_solves(torch, base, steps, 3, refined, stream)
        e1, e2, fl = E.check(base, holder["w"], lr, n)
        it = holder["it"].cpu().numpy()
        ref = {"matrices_per_s": L / ms_r * 1e3, "ms": ms_r, "gate_flags": int((fl != 0).sum()),
               "max_err1": float(e1.max()), "max_err2": float(e2.max()),
               "iterations": np.bincount(it, minlength=4).tolist(), "fallback": int((it == 0).sum())}
        del rwk
        chosen = "refined" if (ref["matrices_per_s"] > plain["matrices_per_s"] and
                               ref["gate_flags"] <= plain["gate_flags"]) else "plain"
        out[f"{fam}_n{n}_f64_L{L}"] = {"plain": plain, "refined": ref, "chosen": chosen,
                                       "chosen_matrices_per_s": max(plain["matrices_per_s"], ref["matrices_per_s"])
                                       if chosen == "refined" else plain["matrices_per_s"]}
        del base
    return out


def make_theta_family(torch, L, n, seed, device, family_seed=2024):
    """The C5 family A(theta) = A0 + sum_j theta_j E_j (j = 1..4): A0 =
    (G + G^T)/sqrt(2n) with G iid N(0,1), E_j = H_j + H_j^T scaled to unit
    Frobenius norm, H_j iid N(0,1) (numpy generator with family_seed), theta
    iid U[-0.1, 0.1] (seed).  Returns (A0, E, A as FP32 L x n x n)."""
    rng = np.random.default_rng(family_seed)
    gm = rng.standard_normal((n, n))
    a0 = (gm + gm.T) / np.sqrt(2.0 * n)
    e = np.empty((4, n, n))
    for j in range(4):
        h = rng.standard_normal((n, n))
        h = h + h.T
        e[j] = h / np.linalg.norm(h)
    th = np.random.default_rng(seed).uniform(-0.1, 0.1, size=(L, 4))
    a = a0[None] + np.einsum("lj,jik->lik", th, e)
    return (torch.from_numpy(a0).to(device), torch.from_numpy(e).to(device),
            torch.from_numpy(np.ascontiguousarray(a.astype(np.float32))).to(device))


def learned_block(torch, E, args, stream, L=65536):
    """C5: L (default 65536) FP32 matrices n = 64 of the theta family.  The
    network is trained (200k solver-generated eigenpairs, the library's own
    kernels; time reported, outside the timed solves), then the learned
    solve is timed against the plain FP32 path and against the same polish
    started from A0's eigenbasis or from the identity (the method without
    the network)."""
    import eigeng_b200.learned as lw
    dev = torch.device("cuda", torch.cuda.current_device())
    n = 64
    a0, e, base = make_theta_family(torch, L, n, 123, dev)
    t0 = time.perf_counter()
    v0 = lw.basis_eigenvectors(a0)
    fam = lw.family_buffer(a0, e, v0)
    x, t = lw.make_dataset(a0, e, v0, 200000, seed=11)
    torch.cuda.synchronize()
    t_data = time.perf_counter() - t0
    net = lw.MLP(512, 512, n * n, seed=5)
    t0 = time.perf_counter()
    hist = lw.train(net, x, t, epochs=args.learned_epochs, batch=1024, lr=1e-3, lr_final=2e-5)
    torch.cuda.synchronize()
    t_train = time.perf_counter() - t0
    del x, t
    steps = max(3, min(args.steps, 10))
    wk = E.workspace(L, n, n, torch.float32, dev)
    w = torch.empty((L, n), dtype=torch.float32, device=dev)
    ms_p, _ = timed_solves(torch, base, steps, 3, lambda a: E.eigen_GPU_batch_ex(a, w, wk, n, stream=stream), stream)
    del wk
    out = {"workload": f"theta family L={L} n={n} f32", "train": {"pairs": 200000, "epochs": args.learned_epochs,
           "data_s": t_data, "train_s": t_train, "mse_first_epoch": hist[0], "mse_last_epoch": hist[-1],
           "widths": list(net.dims)},
           "plain_fp32": {"matrices_per_s": L / ms_p * 1e3, "ms": ms_p}}
    lwk = lw.learned_workspace(L, n, n, net.dims, device=dev)
    for name, warm in (("network", lw.WARM_NETWORK), ("a0_basis", 1), ("identity", 2)):
        holder = {}

        def solve(a):
            holder["r"] = lw.solve_learned(a, n, fam, net if warm == 0 else None, warm=warm, wk=lwk, stream=stream)
        ms, _ = timed_solves(torch, base, steps, 3, solve, stream)
        wv, info, sw, resid = holder["r"]
        swn = sw.cpu().numpy()
        ok = swn >= 0
        rn = resid.cpu().numpy()
        # the residual gate's largest relative residual among the matrices
        # it passed (those it failed, set to infinity there, went to the
        # plain solve and are counted in "fallback")
        out[name] = {"matrices_per_s": L / ms * 1e3, "ms": ms, "gate_pass": float(ok.mean()),
                     "fallback": int((~ok).sum()),
                     "mean_sweeps": float(swn[ok].mean()) if ok.any() else None,
                     "max_gate_residual": float(rn[ok].max()) if ok.any() else None,
                     "info_nonzero": int((info != 0).sum())}
    return out


def run_form(args):
    """One JSON line for the refined or the learned form alone (one GPU),
    same timing rules as the plain solve: fresh copy per step, warm-up, CUDA
    events on the launching stream."""
    import torch
    import eigeng_b200 as E
    torch.cuda.set_device(0)
    stream = torch.cuda.current_stream()
    clk = ClockSampler(0).start()
    try:
        if args.form == "learned":
            w0 = time.perf_counter()
            out = learned_block(torch, E, args, stream, L=args.L)
            w1 = time.perf_counter()
            line = {"metric": f"eigendecomps/s learned form (n=64, f32, theta family, L={args.L})",
                    "value": out["network"]["matrices_per_s"], "unit": "matrices/s", "n_gpus": 1,
                    "higher_is_better": True, "dtype": "f32", "data": "synthetic theta family", "learned": out}
        else:
            n, L = args.n, args.L
            dev = torch.device("cuda", 0)
            base = make_family_batch(torch, args.family, L, n, 4242, dev)
            rwk = E.refine_workspace(L, n, n, device=dev)
            holder = {}

            def refined(a):
                holder["w"], holder["info"], holder["it"] = E.solve_refined(a, n, wk=rwk, stream=stream)
            w0 = time.perf_counter()
            ms, last = timed_solves(torch, base, max(1, args.steps), max(3, args.warmup), refined, stream)
            w1 = time.perf_counter()
            e1, e2, fl = E.check(base, holder["w"], last, n)
            it = holder["it"].cpu().numpy()
            line = {"metric": f"eigendecomps/s refined form (n={n}, f64, {args.family}, L={L})",
                    "value": L / ms * 1e3, "unit": "matrices/s", "n_gpus": 1, "steps": args.steps,
                    "warmup": max(3, args.warmup), "ms_per_step": ms, "higher_is_better": True, "dtype": "f64",
                    "data": "synthetic, seeded on device", "gate_flags": int((fl != 0).sum()),
                    "max_err1": float(e1.max()), "max_err2": float(e2.max()),
                    "iterations": np.bincount(it, minlength=4).tolist(), "fallback": int((it == 0).sum())}
    finally:
        clk.stop()
    line["clocks"] = clk.summary(w0, w1)
    s = json.dumps(line)
    print(s, flush=True)
    if args.out:
        with open(args.out, "a") as f:
            f.write(s + "\n")


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)
    if args.uneven:
        return run_uneven_bench(args)
    if args.impl == "cusolver":
        return run_cusolver(args)
    if args.form != "plain":
        return run_form(args)
    import torch
    import torch.distributed as dist
    import eigeng_b200 as E

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        import datetime
        # short: a rank that fails makes the others' next collective fail too
        dist.init_process_group("nccl", device_id=dev, timeout=datetime.timedelta(seconds=300))

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()

    dt = torch.float64 if args.dtype == "f64" else torch.float32
    esize = 8 if dt == torch.float64 else 4
    n, L = args.n, args.L
    method = {"tql2": E.TQL2, "imtql2": E.IMTQL2, "jacobi": E.JACOBI}[args.method]
    base = make_batch(torch, args.family, L, n, dt, seed=1234 + rank, device=dev)
    inp = FreshInputs(torch, base, args.steps + args.warmup)
    w = torch.empty((L, n), dtype=dt, device=dev)
    info = torch.zeros(L, dtype=torch.int32, device=dev)
    wk = E.workspace(L, n, n, dt, dev) if method != E.JACOBI else None
    stream = torch.cuda.current_stream()

    def solve(a):
        st = E.eigen_GPU_batch_ex(a, w, wk, n, info=info, method=method, stream=stream)
        if st != 0:
            raise RuntimeError(f"solve failed: cudaError {st}")

    clk = ClockSampler(local).start()
    try:
        last = None
        for i in range(args.warmup):
            last = inp.next()
            solve(last)
        if last is None:  # no warm-up: one checked solve outside the count
            last = base.clone()
            solve(last)
        barrier()
        # correctness of the timed configuration: the reference's gate on the
        # last warm-up solve
        e1, e2, fl = E.check(base, w, last, n)
        torch.cuda.synchronize()
        gate_fail = int((fl != 0).sum().item())
        info_fail = int((info != 0).sum().item())

        t0 = torch.cuda.Event(enable_timing=True)
        t1 = torch.cuda.Event(enable_timing=True)
        barrier()
        w0 = time.perf_counter()
        t0.record(stream)
        for i in range(args.steps):
            solve(inp.next())
        t1.record(stream)
        barrier()
        w1 = time.perf_counter()
    finally:
        clk.stop()
    ms = t0.elapsed_time(t1)
    if world > 1:
        tt = torch.tensor([ms], dtype=torch.float64, device=dev)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        ms = float(tt.item())
    value = world * L * args.steps / (ms / 1000.0)
    l2_note = inp.note()
    del inp, last

    # per-phase kernel times on the launching stream (extra traced solves,
    # up to ten, same inputs as the timed region)
    phases, nchunks = [], 1
    for i in range(min(args.steps, 10)):
        a = base.clone()
        with E.PhaseTrace(chunks=64) as tr:
            solve(a)
        per_chunk = tr.ms()
        nchunks = max(1, len(per_chunk))
        phases.append(np.array(per_chunk).sum(axis=0))  # workspace chunks run one after another
    ph = np.array(phases).mean(axis=0) if phases else np.zeros(3)
    hbm, peak_kind = peaks()

    # record counts (mean rotations per matrix) for the algorithmic byte model
    recs = 1.1 * n * n
    pb = phase_bytes(n, esize, recs)
    names = ["tridiag_qt", "ql_rotations", "apply_rotations"]
    dom = int(np.argmax(ph))
    achieved = pb[dom] * L / (ph[dom] / 1000.0) / 1e9 if ph[dom] > 0 else 0.0
    traffic = measured_traffic(names[dom], args.dtype, n)

    line = {
        "metric": f"eigendecomps/s (n={n}, {args.dtype}, {args.family}, L={L})",
        "value": value, "unit": "matrices/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": args.dtype, "data": "synthetic, seeded on device: " + FAMILY_TEXT[args.family],
        "config": workload_config(args, world, l2_note),
        "gpu_launches": 3 * nchunks * args.steps,
        "correctness": {"reference_gate_flags": gate_fail, "info_nonzero": info_fail,
                        "max_err1": float(e1.max().item()), "max_err2": float(e2.max().item())},
        "phases_ms": {k: float(v) for k, v in zip(names, ph)},
        "roofline": {"bound": "hbm", "kernel": names[dom], "achieved": achieved, "peak": hbm, "unit": "GB/s",
                     "frac": achieved / hbm, "peak_kind": peak_kind,
                     "traffic": traffic * L if traffic else None,
                     "traffic_source": "profiles/dram_traffic.txt (ncu DRAM bytes per matrix at 2-4x L2 inputs, x L)"
                     if traffic else None,
                     "alg_bytes_per_matrix": pb[dom]},
        "hbm_fraction_whole_solve": alg_bytes(n, esize) * value / world / 1e9 / hbm,
        "clocks": clk.summary(w0, w1),
    }

    if not args.no_e2e:
        # end to end through the public host-buffer call (eigeng_b200.solve_host):
        # every step copies A in from pinned host memory, solves, and copies
        # the eigenvectors and eigenvalues back, the copies of one chunk
        # overlapping the solve of another
        host_in = base.cpu().pin_memory()
        host_out = torch.empty_like(host_in).pin_memory()
        host_w = torch.empty((L, n), dtype=dt).pin_memory()
        for _ in range(2):
            E.solve_host(host_in, n, w_host=host_w, z_host=host_out, method=method, stream=stream)
        barrier()
        e0 = torch.cuda.Event(enable_timing=True)
        e1_ = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(args.steps):
            E.solve_host(host_in, n, w_host=host_w, z_host=host_out, method=method, stream=stream)
        e1_.record(stream)
        barrier()
        ems = e0.elapsed_time(e1_)
        if world > 1:
            tt = torch.tensor([ems], dtype=torch.float64, device=dev)
            dist.all_reduce(tt, op=dist.ReduceOp.MAX)
            ems = float(tt.item())
        line["e2e"] = {"value": world * L * args.steps / (ems / 1000.0), "unit": "matrices/s",
                       "h2d_bytes_per_step": L * n * n * esize, "d2h_bytes_per_step": L * n * n * esize + L * n * esize}

    if not args.no_extra:
        # the metric's other sizes, same timing rules (fresh copy per step,
        # warm-up, CUDA events on the launching stream, max over ranks)
        sizes = {}
        for n2, L2 in ((32, 16384), (256, 2048)):
            if n2 == n and dt == torch.float64:
                continue
            b2 = make_batch(torch, "symu", L2, n2, torch.float64, seed=99 + rank, device=dev)
            cps = FreshInputs(torch, b2, args.steps + args.warmup)
            w2 = torch.empty((L2, n2), dtype=torch.float64, device=dev)
            wk2 = E.workspace(L2, n2, n2, torch.float64, dev)
            for i in range(args.warmup):
                E.eigen_GPU_batch_ex(cps.next(), w2, wk2, n2, stream=stream)
            barrier()
            f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            f0.record(stream)
            for i in range(args.steps):
                E.eigen_GPU_batch_ex(cps.next(), w2, wk2, n2, stream=stream)
            f1.record(stream)
            barrier()
            ms2 = f0.elapsed_time(f1)
            if world > 1:
                tt = torch.tensor([ms2], dtype=torch.float64, device=dev)
                dist.all_reduce(tt, op=dist.ReduceOp.MAX)
                ms2 = float(tt.item())
            sizes[f"n{n2}_f64_L{L2}"] = world * L2 * args.steps / (ms2 / 1000.0)
            del cps, wk2
        line["sizes"] = {"unit": "matrices/s", "data": "synthetic (B + B^T)/2, B iid U[-1,1]", **sizes}

    if not args.no_extra and world == 1:
        line["gate_in_packed_solve"] = gate_in_packed_solve(torch, E, base, n, stream, max(3, min(args.steps, 10)))
    if not args.no_chosen and world == 1:
        line["chosen_vs_plain"] = chosen_vs_plain(torch, E, args, stream)
    if not args.no_learned and world == 1:
        line["learned"] = learned_block(torch, E, args, stream)

    if rank == 0 and world == 1 and not args.no_cpu:  # the CPU baseline is an N=1 figure
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import oracle as O
        nth = os.cpu_count() or 1
        sample = base[:min(L, CPU_SAMPLE)].cpu().numpy().reshape(-1, n, n)
        r, cnt, el = cpu_time_oracle(sample, n, {"tql2": 0, "imtql2": 1, "jacobi": 2}[args.method], 10.0, nth)
        line["cpu_baseline"] = {"value": r, "unit": "matrices/s", "cores": nth, "kind": "port",
                                "sample": f"{sample.shape[0]} matrices of the workload re-solved {cnt // sample.shape[0]}x "
                                          f"in {el:.1f} s"}

    if rank == 0:
        s = json.dumps(line)
        print(s, flush=True)
        if args.out:
            with open(args.out, "a") as f:
                f.write(s + "\n")
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
