"""Train the flexure warm-start U-Net on the device and report what it gains.

    python deep-time_b200/train_unet.py --samples 20000 --heldout 2000 --epochs 50 \
        --out deep-time_b200/weights/unet_flexure.bin

Data: seeded (q, log10 D) pairs on the 512 x 256, dx = 10 km raster (rigidity smoothed over 8
cells), labelled by this library's FP64 PCG to a relative residual of 1e-10. Model: the library's
U-Net (4 levels, 32 base channels, 3 x 3 convolutions, BF16, FP32 accumulation), Adam at lr 1e-3
on the MSE of the deflection normalised by rms(q) / (delta-rho g). The held-out report gives the
first guess's relative residual ||b - A w0|| / ||b|| (the zero guess's is 1) and the PCG
iterations to 1e-10 with and without it.
"""
import argparse
import ctypes
import json
import os
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)

import numpy as np  # noqa: E402


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--samples", type=int, default=20000)
    ap.add_argument("--heldout", type=int, default=2000)
    ap.add_argument("--epochs", type=int, default=50)
    ap.add_argument("--batch", type=int, default=16)
    ap.add_argument("--lr", type=float, default=1e-3)
    ap.add_argument("--out", default=os.path.join(HERE, "weights", "unet_flexure.bin"))
    ap.add_argument("--report", default=None)
    ap.add_argument("--eval-solves", type=int, default=200, help="held-out samples solved with and without the guess")
    args = ap.parse_args()

    import torch

    from deeptime_gpu import _lib as L
    from deeptime_gpu import flexure as F
    from deeptime_gpu import unet as U

    def log(msg):
        print(msg, flush=True)

    w, h, dx = 512, 256, 10_000.0
    t0 = time.time()
    X, T, its, rels = U.make_dataset(args.samples, w, h, dx, log=log)
    t_data = time.time() - t0
    log(f"data: {args.samples} pairs in {t_data:.1f} s; label PCG iterations mean {np.mean(its):.1f}, "
        f"max rel. residual {max(rels):.2e}")
    ntr = args.samples - args.heldout
    model = U.UNet(seed=20261203)
    t0 = time.time()
    hist = U.train(model, X[:ntr], T[:ntr], epochs=args.epochs, batch=args.batch, lr=args.lr, log=log)
    t_train = time.time() - t0
    os.makedirs(os.path.dirname(args.out), exist_ok=True)
    model.save(args.out)
    log(f"training: {args.epochs} epochs in {t_train:.1f} s, final loss {hist[-1]:.5f}; weights -> {args.out}")

    # held-out: the first guess's residual and the iterations it saves
    lib = L.lib()
    sv = F.Solver(w, h, dx)
    L.check(lib.dt_flex_set_unet(sv._h, model._h, ctypes.c_double(dx)))
    dev = torch.device("cuda")
    x_dev = torch.zeros((h, w), dtype=torch.float64, device=dev)
    first_rel, its_cold, its_warm = [], [], []
    seed0 = 50_000
    for k in range(ntr, args.samples):
        d, c, b = U.flexure_problem_torch(w, h, 8.0, seed0 + 2 * k, dev)
        torch.cuda.synchronize()
        rep = L.Report()
        p = F.params(precond=L.PRECOND_REFERENCE, stop=L.STOP_REL_RESIDUAL, tol=1e-10, max_iterations=0,
                     warm_start=L.WARM_UNET)
        st = lib.dt_flex_solve_dev(sv._h, ctypes.c_void_p(d.data_ptr()), ctypes.c_void_p(c.data_ptr()),
                                   ctypes.c_void_p(b.data_ptr()), ctypes.c_void_p(x_dev.data_ptr()), ctypes.byref(p),
                                   ctypes.byref(rep))
        L.check(st, allow=(L.DT_OK, L.DT_NOT_CONVERGED))
        first_rel.append(rep.warm_start_rel_residual)
        if k - ntr < args.eval_solves:
            for warm, out in ((L.WARM_NONE, its_cold), (L.WARM_UNET, its_warm)):
                p = F.params(precond=L.PRECOND_REFERENCE, stop=L.STOP_REL_RESIDUAL, tol=1e-10, max_iterations=5000,
                             warm_start=warm)
                st = lib.dt_flex_solve_dev(sv._h, ctypes.c_void_p(d.data_ptr()), ctypes.c_void_p(c.data_ptr()),
                                           ctypes.c_void_p(b.data_ptr()), ctypes.c_void_p(x_dev.data_ptr()),
                                           ctypes.byref(p), ctypes.byref(rep))
                L.check(st)
                out.append(rep.iterations)
    first_rel = np.array(first_rel)
    report = {
        "samples": args.samples, "heldout": args.heldout, "epochs": args.epochs, "batch": args.batch, "lr": args.lr,
        "raster": f"{w}x{h}", "dx_m": dx, "data_seconds": t_data, "train_seconds": t_train,
        "label_iterations_mean": float(np.mean(its)), "label_rel_residual_max": float(max(rels)),
        "loss_first_epoch": hist[0], "loss_last_epoch": hist[-1], "loss_history": hist,
        "heldout_first_guess_rel_residual": {"mean": float(first_rel.mean()), "median": float(np.median(first_rel)),
                                             "max": float(first_rel.max()), "zero_guess": 1.0},
        "heldout_pcg_iterations_to_1e-10": {"zero_guess_mean": float(np.mean(its_cold)),
                                             "unet_guess_mean": float(np.mean(its_warm)), "solves": len(its_cold)},
        "params": int(model.n_params),
    }
    log(json.dumps({k: v for k, v in report.items() if k != "loss_history"}))
    path = args.report or os.path.splitext(args.out)[0] + ".json"
    with open(path, "w") as f:
        json.dump(report, f, indent=1)


if __name__ == "__main__":
    main()
