"""Learned vertical closure: data, training and deployment.

1. Samples: the estuary channel (100 x 20 grid, 10 layers) run with MY2.5 under 8 seeds
   of random wind (speed uniform 0-12 m/s, random heading) and tidal phase; after a
   spin-up, VDIF_Q's inputs and outputs are sampled (``fvg_closure_sample``) at every
   interior level of every wet node until the requested number of samples is reached.
2. Scaling: inputs [N^2, S^2, D, sigma, u*_surf, u*_bot, q2, q2l] -> asinh(x/s) for the
   signed and heavy-tailed ones (N^2, S^2, u*), log for D, q2, q2l, identity for sigma;
   then standardised.  Targets (KN*KAPPA*SM, KN*SM, KN*SH*VPRNU, all >= 0) ->
   log(y + eps), standardised.  The envelope is the 0.5 and 99.5 percentiles of every raw
   input over the training samples.
3. Training: ``fvg_mlp_train`` (the library's CUDA forward/backward kernels, Adam).
4. Deployment: ``attach(model, trained)`` -> ``fvg_set_closure``: BF16 tensor-core
   inference in the closure step, MY2.5 for every column outside the envelope.
"""
from __future__ import annotations

import numpy as np

FEATURES = ("N2", "S2", "D", "sigma", "ustar_surf", "ustar_bot", "q2", "q2l")
TARGETS = ("kq_new", "km_new", "kh_new")
KIND = (2, 2, 1, 0, 2, 2, 1, 1)          # 0 identity, 1 log, 2 asinh(x/scale)
TEPS = 1e-9


def channel_seed_case(seed, base_kw=None):
    """The estuary channel with a seeded wind and tidal phase."""
    from . import cases
    rng = np.random.default_rng(1000 + seed)
    speed = rng.uniform(0.0, 12.0)
    head = rng.uniform(0.0, 2 * np.pi)
    phase = rng.uniform(0.0, 360.0)
    c = cases.estuary_channel(**(base_kw or {}))
    c["forcing"]["tide"]["phai"] = c["forcing"]["tide"]["phai"] + phase
    c["forcing"]["wind"] = {"kind": "speed", "u": speed * np.cos(head), "v": speed * np.sin(head)}
    c["name"] = c["name"] + "-seed%d" % seed
    return c


def coastal_seed_case(seed, npts=50000, kb=41):
    """The coastal mesh (default 50k nodes, 40 layers) with a seeded wind and tidal phase."""
    from . import cases
    rng = np.random.default_rng(2000 + seed)
    speed = rng.uniform(0.0, 12.0)
    head = rng.uniform(0.0, 2 * np.pi)
    phase = rng.uniform(0.0, 360.0)
    c = cases.coastal_mesh(npts=npts, kb=kb, wind_speed=speed)
    c["forcing"]["tide"]["phai"] = c["forcing"]["tide"]["phai"] + phase
    c["forcing"]["wind"] = {"kind": "speed", "u": speed * np.cos(head), "v": speed * np.sin(head)}
    c["name"] = c["name"] + "-seed%d" % seed
    return c


def generate(n_target=5_000_000, seeds=8, spinup=360, every=5, base_kw=None, source="channel"):
    """(X [n,8], Y [n,3]) float32 samples of MY2.5 from seeded runs of the estuary channel
    (``source`` "channel", the training set of the closure as specified) or of the 50k-node
    coastal mesh ("coastal")."""
    import ctypes as C
    import torch
    from .engine import Fvcom
    per_seed = int(np.ceil(n_target / seeds))
    xs, ys = [], []
    for sd in range(seeds):
        case = channel_seed_case(sd, base_kw) if source == "channel" else coastal_seed_case(sd)
        f = Fvcom(case)
        M, K = f.M, f.KB - 1
        S = M * (K - 1)
        buf = torch.zeros(12 * S, dtype=torch.float32, device="cuda")
        f.run(spinup)
        got = 0
        while got < per_seed:
            f.run(every - 1)
            f.lib.fvg_closure_sample.argtypes = [C.c_void_p, C.c_void_p, C.c_int64]
            f._check(f.lib.fvg_closure_sample(f.h, buf.data_ptr(), buf.numel()), "fvg_closure_sample")
            f.run(1)
            f.lib.fvg_closure_sample(f.h, None, 0)
            a = buf.view(12, S).cpu().numpy()
            wet = a[11] > 0.5
            x = a[:8, wet].T
            y = a[8:11, wet].T
            ok = np.isfinite(x).all(axis=1) & np.isfinite(y).all(axis=1)
            xs.append(x[ok])
            ys.append(y[ok])
            got += int(ok.sum())
        f.close()
    X = np.concatenate(xs)[:n_target].astype(np.float32)
    Y = np.concatenate(ys)[:n_target].astype(np.float32)
    return X, Y


def fit_scaling(X, Y):
    """Scaling vector of fvg_set_closure (55 floats) from training samples."""
    scale = np.ones(8, dtype=np.float64)
    for f, k in enumerate(KIND):
        if k == 2:
            med = np.median(np.abs(X[:, f]))
            scale[f] = med if med > 0 else 1.0
    T = transform_x(X, scale)
    mean = T.mean(axis=0)
    std = T.std(axis=0)
    std[std == 0] = 1.0
    lo = np.percentile(X, 0.5, axis=0)
    hi = np.percentile(X, 99.5, axis=0)
    ty = np.log(Y.astype(np.float64) + TEPS)
    tmean, tstd = ty.mean(axis=0), ty.std(axis=0)
    tstd[tstd == 0] = 1.0
    return np.concatenate([np.array(KIND, dtype=np.float64), scale, mean, std, lo, hi, tmean, tstd,
                           [TEPS]]).astype(np.float32)


def _parts(norm):
    n = np.asarray(norm, dtype=np.float64)
    return dict(kind=n[0:8].astype(int), scale=n[8:16], mean=n[16:24], std=n[24:32], lo=n[32:40],
                hi=n[40:48], tmean=n[48:51], tstd=n[51:54], teps=n[54])


def transform_x(X, scale):
    X = np.asarray(X, dtype=np.float64)
    T = np.empty_like(X)
    for f, k in enumerate(KIND):
        if k == 0:
            T[:, f] = X[:, f]
        elif k == 1:
            T[:, f] = np.log(np.maximum(X[:, f], 1e-30))
        else:
            T[:, f] = np.arcsinh(X[:, f] / scale[f])
    return T


def normalise(X, Y, norm):
    p = _parts(norm)
    xn = (transform_x(X, p["scale"]) - p["mean"]) / p["std"]
    yn = (np.log(np.asarray(Y, dtype=np.float64) + p["teps"]) - p["tmean"]) / p["tstd"]
    return xn.astype(np.float32), yn.astype(np.float32)


def denormalise_y(yn, norm):
    p = _parts(norm)
    return np.maximum(np.exp(np.asarray(yn, dtype=np.float64) * p["tstd"] + p["tmean"]) - p["teps"], 0.0)


def inside(X, norm):
    p = _parts(norm)
    return np.all((X >= p["lo"]) & (X <= p["hi"]), axis=1)


def train(X, Y, epochs=12, batch=4096, lr=2e-3, seed=0):
    """Train on the device; returns {"params", "norm", "history"}."""
    import torch
    from .engine import Mlp
    norm = fit_scaling(X, Y)
    xn, yn = normalise(X, Y, norm)
    dx = torch.from_numpy(xn).cuda()
    dy = torch.from_numpy(yn).cuda()
    net = Mlp(seed=seed)
    hist = net.train(dx.data_ptr(), dy.data_ptr(), xn.shape[0], epochs, batch, lr, seed=seed)
    params = net.params()
    net.close()
    return {"params": params, "norm": norm, "history": hist}


def predict(trained, X):
    """FP32 network prediction of the new parts for raw inputs X (device forward pass)."""
    import torch
    from .engine import Mlp
    xn, _ = normalise(X, np.ones((X.shape[0], 3), dtype=np.float32), trained["norm"])
    net = Mlp()
    net.set_params(trained["params"])
    dx = torch.from_numpy(xn).cuda()
    out = torch.zeros((X.shape[0], 3), dtype=torch.float32, device="cuda")
    net.forward(dx.data_ptr(), X.shape[0], out.data_ptr())
    net.close()
    return denormalise_y(out.cpu().numpy(), trained["norm"])


def attach(model, trained):
    """Switch ``model`` (engine.Fvcom) to the learned closure."""
    import ctypes as C
    p = np.ascontiguousarray(trained["params"], dtype=np.float32)
    n = np.ascontiguousarray(trained["norm"], dtype=np.float32)
    fp = C.POINTER(C.c_float)
    model.lib.fvg_set_closure.argtypes = [C.c_void_p, C.c_int32, fp, C.c_int32, fp, C.c_int32]
    rc = model.lib.fvg_set_closure(model.h, 1, p.ctypes.data_as(fp), p.size, n.ctypes.data_as(fp), n.size)
    model._check(rc, "fvg_set_closure")


def detach(model):
    import ctypes as C
    model.lib.fvg_set_closure.argtypes = [C.c_void_p, C.c_int32, C.c_void_p, C.c_int32, C.c_void_p, C.c_int32]
    model._check(model.lib.fvg_set_closure(model.h, 0, None, 0, None, 0), "fvg_set_closure")


def status(model):
    import ctypes as C
    a, b = C.c_int32(), C.c_int32()
    model.lib.fvg_closure_status.argtypes = [C.c_void_p, C.POINTER(C.c_int32), C.POINTER(C.c_int32)]
    model._check(model.lib.fvg_closure_status(model.h, C.byref(a), C.byref(b)), "fvg_closure_status")
    return {"columns_on_network": a.value, "wait_timeouts": b.value}


def save(trained, path):
    np.savez_compressed(path, params=trained["params"], norm=trained["norm"], history=trained["history"])


def load(path):
    d = np.load(path)
    return {"params": d["params"], "norm": d["norm"], "history": d["history"]}


def evaluate_on(case, trained, steps=200, precision="fp64"):
    """Run ``case`` with MY2.5 and with the learned closure for ``steps`` internal steps from
    the same cold start; errors of the learned run and the closure-step device times."""
    import ctypes as C
    from .engine import Fvcom
    from .precision_report import compare

    def group_ms(f, name, n=2):
        L = f.lib
        L.fvg_profile.argtypes = [C.c_void_p, C.c_int32, C.POINTER(C.c_double), C.POINTER(C.c_double)]
        L.fvg_profile_groups.restype = C.c_int32
        L.fvg_profile_group_name.restype = C.c_char_p
        L.fvg_profile_group_name.argtypes = [C.c_int32]
        ng = L.fvg_profile_groups()
        g = (C.c_double * ng)()
        tot = C.c_double()
        L.fvg_profile(f.h, n, g, C.byref(tot))
        names = [L.fvg_profile_group_name(i).decode() for i in range(ng)]
        return g[names.index(name)] / n, tot.value / n

    a, b = Fvcom(case), Fvcom(case)
    a.set_precision(precision)
    b.set_precision(precision)
    attach(b, trained)
    a.run(steps)
    b.run(steps)
    st = status(b)
    err = compare(a, b)
    km_a, km_b = a.get3("km")[1:, 1:-1], b.get3("km")[1:, 1:-1]
    err["KM_rel_rms"] = float(np.sqrt(np.mean((km_a - km_b) ** 2)) / np.sqrt(np.mean(km_a ** 2)))
    va, sa = group_ms(a, "vdif_q")
    vb, sb = group_ms(b, "vdif_q")
    vb += group_ms(b, "closure")[0]  # the network kernel, its own profile group
    out = {"steps": steps, "errors_vs_my25": err, "columns_on_network": st["columns_on_network"],
           "nodes": case["grid"]["M"], "wait_timeouts": st["wait_timeouts"],
           "closure_step_ms": {"my25": va, "learned": vb}, "step_ms": {"my25": sa, "learned": sb}}
    a.close()
    b.close()
    return out


def main():
    import argparse
    import json
    import time
    ap = argparse.ArgumentParser(description="train the learned closure and evaluate it")
    ap.add_argument("--samples", type=int, default=5_000_000)
    ap.add_argument("--epochs", type=int, default=12)
    ap.add_argument("--batch", type=int, default=4096)
    ap.add_argument("--lr", type=float, default=2e-3)
    ap.add_argument("--out", default=None, help="write the trained network (.npz)")
    ap.add_argument("--eval-npts", type=int, default=200000)
    ap.add_argument("--eval-steps", type=int, default=200)
    ap.add_argument("--source", default="channel", choices=["channel", "coastal"])
    ap.add_argument("--load", default=None,
                    help="evaluate a trained network (.npz from --out) instead of generating and training one")
    args = ap.parse_args()
    from . import cases
    if args.load:
        trained = load(args.load)
        report = {"network": args.load,
                  "coastal": evaluate_on(cases.coastal_mesh(npts=args.eval_npts), trained, args.eval_steps)}
        print(json.dumps(report))
        return
    t0 = time.time()
    X, Y = generate(args.samples, source=args.source)
    t1 = time.time()
    rng = np.random.default_rng(0)
    perm = rng.permutation(X.shape[0])
    nh = X.shape[0] // 10
    hold, tr_i = perm[:nh], perm[nh:]
    trained = train(X[tr_i], Y[tr_i], epochs=args.epochs, batch=args.batch, lr=args.lr)
    t2 = time.time()
    inside_h = inside(X[hold], trained["norm"])
    pred = predict(trained, X[hold][inside_h])
    ref = Y[hold][inside_h]
    rel = np.abs(pred - ref) / (np.abs(ref) + 1e-7)
    report = {"source": args.source, "samples": int(X.shape[0]), "generate_s": t1 - t0, "train_s": t2 - t1,
              "history": [float(h) for h in trained["history"]],
              "holdout": {"inside_envelope": float(inside_h.mean()),
                          "median_rel_err": [float(v) for v in np.median(rel, axis=0)],
                          "p90_rel_err": [float(v) for v in np.percentile(rel, 90, axis=0)]}}
    if args.out:
        save(trained, args.out)
    if args.eval_npts:
        report["coastal"] = evaluate_on(cases.coastal_mesh(npts=args.eval_npts), trained, args.eval_steps)
    print(json.dumps(report))


if __name__ == "__main__":
    main()
