"""Times the reference's own GPU build on this GPU -- TEST INFRASTRUCTURE.

A reported baseline, never part of the product: loads
oracle/_ref/libeigenGbatch_ref.so (the reference's eigen_GPU_batch.cu built
for sm_100a by oracle/build_ref.sh) and calls its stock C entry points
exactly as its README documents them (size query with wk == NULL, then the
solve, eigen_GPU_batch.h:26-30), on the same seeded batches and under the
same timing rules as bench.py's own arm: a pristine device copy per step,
W warm-up steps, K timed steps between CUDA events on the launching stream,
inputs larger than L2.  Prints one JSON line per configuration.

    python oracle/time_ref_gpu.py [--steps K] [--warmup W] [--out FILE]
"""
import argparse
import ctypes
import json
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

REF_LIB = os.path.join(ROOT, "oracle", "_ref", "libeigenGbatch_ref.so")

# (family, n, L, dtype): the metric's sizes and the headline configuration
CONFIGS = [("symu", 32, 16384, "f64"), ("letkf", 128, 4096, "f64"), ("symu", 256, 2048, "f64"),
           ("symu", 32, 16384, "f32"), ("letkf", 128, 4096, "f32"), ("symu", 256, 2048, "f32")]


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--out", default=None)
    args = ap.parse_args()
    import torch
    import bench as B

    lib = ctypes.CDLL(REF_LIB)
    dev = torch.device("cuda", 0)
    stream = torch.cuda.current_stream(dev)
    for fam, n, L, dts in CONFIGS:
        dt = torch.float64 if dts == "f64" else torch.float32
        fn = lib.eigen_GPU_batch_DP if dt == torch.float64 else lib.eigen_GPU_batch_FP
        fn.restype = None
        fn.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p,
                       ctypes.c_void_p, ctypes.c_void_p]
        lw = ctypes.c_size_t(0)
        fn(L, n, n, n, None, ctypes.addressof(lw), None, None)
        base = B.make_batch(torch, fam, L, n, dt, seed=1234, device=dev)
        inp = B.FreshInputs(torch, base, args.steps + args.warmup)
        w = torch.empty((L, n), dtype=dt, device=dev)
        wk = torch.empty(max(lw.value, 16), dtype=torch.uint8, device=dev)

        def solve(a):
            fn(L, n, n, n, a.data_ptr(), w.data_ptr(), wk.data_ptr(), stream.cuda_stream)

        last = None
        for _ in range(args.warmup):
            last = inp.next()
            solve(last)
        torch.cuda.synchronize()
        import eigeng_b200 as E  # noqa: the library's own gate kernel checks the reference's output
        e1, e2, fl = E.check(base, w, last, n)
        e0, e1_ = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(args.steps):
            solve(inp.next())
        e1_.record(stream)
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1_) / args.steps
        line = {"impl": "reference-gpu", "library": "oracle/_ref/libeigenGbatch_ref.so (tql2 + DO_SORT, sm_100a)",
                "metric": f"eigendecomps/s (n={n}, {dts}, {fam}, L={L})", "value": L / (ms / 1000.0),
                "unit": "matrices/s", "ms_per_step": ms, "steps": args.steps, "warmup": args.warmup,
                "workspace_bytes": lw.value, "config": {"workload": f"{fam} L={L} n={n} {dts} tql2 sorted",
                                                        "l2_flush": inp.note()},
                "reference_gate_flags": int((fl != 0).sum().item()), "max_err1": float(e1.max().item()),
                "max_err2": float(e2.max().item())}
        print(json.dumps(line), flush=True)
        if args.out:
            with open(args.out, "a") as f:
                f.write(json.dumps(line) + "\n")
        del inp, base, wk


if __name__ == "__main__":
    main()
