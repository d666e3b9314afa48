"""Learned sub-grid closure: decaying homogeneous isotropic turbulence (HIT),
the fine plain-LBM run that generates training data, the trainer and the
coarse runs it is judged on.

    python -m lbm.closure run [--fine 512] [--factor 4] [--snapshots 2000] ...

(run from gpu-sims_b200/, or with it on sys.path) prints one JSON line with
the spectra errors of the coarse Smagorinsky and learned-closure runs
against the box-filtered fine run, and the wall times of the runs.

The pipeline (all compute in the library's kernels; torch only holds device
memory, generates the seeded initial field and evaluates spectra):
  1. seeded solenoidal initial velocity, E(k) ~ k^4 exp(-2 (k/k0)^2), k0 = 4,
     scaled to u_rms = 0.04 per component, rho = 1;
  2. fine periodic plain-BGK run; every `every` fine steps the moments are
     box-filtered by `factor` (lbm_box_filter) and `samples_per_snapshot`
     training samples drawn from the filtered field (lbm_closure_samples):
     9 features of the non-equilibrium flux, the target Cs^2 ratio
     r = -tau^d:S / (Cs0^2 |S|^3) and weight |S|^3;
  3. the MLP (9 -> 32 -> 32 -> 1, softplus output) trained by the fused
     forward/backward and Adam kernels (lbm_trainer_fit);
  4. coarse runs from the filtered initial field, dt_c = factor dt_f,
     tau_c = 1/2 + (tau_f - 1/2)/factor: Smagorinsky Cs0 and the learned
     closure (Cs^2 = Cs0^2 r per node, fused in the collide);
  5. shell-averaged spectra E(k) of the coarse runs against the filtered fine
     field at matching times.
"""
from __future__ import annotations

import math

import numpy as np


def hit_velocity(n: int, seed: int = 5, u_rms: float = 0.04, k0: float = 4.0, device="cuda"):
    """Seeded solenoidal random velocity on an n^3 periodic grid (torch
    tensor [3][n][n][n], index [c][z][y][x]): Gaussian Fourier coefficients
    projected on the plane normal to k, with shell energy
    E(k) ~ k^4 exp(-2 (k/k0)^2), then scaled so every component has rms
    u_rms."""
    import torch
    g = torch.Generator(device=device).manual_seed(seed)
    k = torch.fft.fftfreq(n, d=1.0 / n, device=device)
    kr = torch.fft.rfftfreq(n, d=1.0 / n, device=device)
    kz, ky, kx = torch.meshgrid(k, k, kr, indexing="ij")
    k2 = kx * kx + ky * ky + kz * kz
    kk = torch.sqrt(k2)
    # per-mode amplitude: E(k) spread over the shell area 4 pi k^2
    amp = torch.where(k2 > 0, kk * torch.exp(-((kk / k0) ** 2)) / math.sqrt(4 * math.pi), 0.0)
    shape = kx.shape
    xi = [torch.complex(torch.randn(shape, generator=g, device=device),
                        torch.randn(shape, generator=g, device=device)) for _ in range(3)]
    kd = (kx * xi[0] + ky * xi[1] + kz * xi[2]) / torch.where(k2 > 0, k2, 1.0)
    u = torch.empty((3, n, n, n), dtype=torch.float32, device=device)
    for c, kc in enumerate((kx, ky, kz)):
        uh = amp * (xi[c] - kc * kd)
        u[c] = torch.fft.irfftn(uh, s=(n, n, n), dim=(0, 1, 2))
        del uh
    del xi, kd, amp, kx, ky, kz, k2, kk
    for c in range(3):
        u[c] *= u_rms / torch.sqrt(torch.mean(u[c].double() ** 2)).float()
    return u


def spectrum(u, kmax: int | None = None) -> np.ndarray:
    """Shell-averaged kinetic-energy spectrum of a periodic velocity field
    (tensor [3][n][n][n]): E[k] = sum over |k'| in [k - 1/2, k + 1/2) of
    |u_hat(k')|^2 / 2, normalised so sum_k E[k] = <|u|^2> / 2."""
    import torch
    n = u.shape[-1]
    k = torch.fft.fftfreq(n, d=1.0 / n, device=u.device)
    kz, ky, kx = torch.meshgrid(k, k, k, indexing="ij")
    shell = torch.round(torch.sqrt(kx * kx + ky * ky + kz * kz)).long().reshape(-1)
    nb = int(shell.max().item()) + 1
    e = torch.zeros(nb, dtype=torch.float64, device=u.device)
    for c in range(3):
        uh = torch.fft.fftn(u[c].double()) / float(n) ** 3
        e.index_add_(0, shell, (0.5 * (uh.real ** 2 + uh.imag ** 2)).reshape(-1))
    e = e.cpu().numpy()
    return e if kmax is None else e[: kmax + 1]


def spectrum_np(u3: np.ndarray, n: int, kmax: int | None = None) -> np.ndarray:
    """spectrum() of a host velocity field u3 [n^3][3] (x-fastest)."""
    import torch
    u = torch.from_numpy(np.ascontiguousarray(u3.T.reshape(3, n, n, n)))
    if torch.cuda.is_available():
        u = u.cuda()
    return spectrum(u, kmax)


def init_net(seed: int, mean: np.ndarray, iscale: np.ndarray) -> np.ndarray:
    """He-initialised network whose output starts near 1 (plain
    Smagorinsky): small last layer, b3 = softplus^-1(1)."""
    import lbm
    rng = np.random.default_rng(seed)
    w = np.zeros(lbm.CLOSURE_FLOATS, np.float32)
    nin, nh = lbm.CLOSURE_INPUTS, lbm.CLOSURE_HIDDEN
    o = 0
    w[o:o + nh * nin] = rng.standard_normal(nh * nin) * math.sqrt(2.0 / nin)
    o += nh * nin + nh
    w[o:o + nh * nh] = rng.standard_normal(nh * nh) * math.sqrt(2.0 / nh)
    o += nh * nh + nh
    w[o:o + nh] = 0.1 * rng.standard_normal(nh) * math.sqrt(1.0 / nh)
    o += nh
    w[o] = math.log(math.e - 1.0)
    o += 1
    w[o:o + nin] = mean
    w[o + nin:o + 2 * nin] = iscale
    return w


def _events():
    import torch
    return torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)


def _coarse_run(lbm, stream, nc, tau_c, cs0, rho0, u0, steps, eval_every, net=None):
    """Coarse periodic BGK-Smagorinsky run (learned closure when net is
    given) from host moments; returns (device seconds of the steps, spectra
    at every eval_every steps, kinetic energy there)."""
    import torch
    d = lbm.default_desc(nx=nc, ny=nc, nz=nc, mode=lbm.MODE_PHYSICS, precision=lbm.PREC_F32,
                         collision=lbm.COLL_BGK, tau=tau_c, periodic=(1, 1, 1), smagorinsky_cs=cs0)
    lat = lbm.Lattice(d)
    lat.set_stream(stream.cuda_stream)
    if net is not None:
        lat.set_closure(net)
    lat.init_from_moments(rho0, u0)
    secs, spectra, ke = 0.0, {}, {}
    ok = True
    for s in range(0, steps, eval_every):
        e0, e1 = _events()
        e0.record(stream)
        lat.step(eval_every)
        e1.record(stream)
        try:
            lat.sync()
        except lbm.LbmError:
            ok = False
            break
        torch.cuda.synchronize()
        secs += e0.elapsed_time(e1) / 1e3
        _, u = lat.read_moments()
        spectra[s + eval_every] = spectrum_np(u, nc)
        ke[s + eval_every] = float(0.5 * np.mean(np.sum(u.astype(np.float64) ** 2, axis=1)))
    lat.close()
    return {"device_s": secs, "spectra": spectra, "ke": ke, "finite": ok}


def run(fine: int = 512, factor: int = 4, tau_f: float = 0.508, snapshots: int = 2000,
        every: int = 8, samples_per_snapshot: int = 4096, cs0: float = 0.1, seed: int = 5,
        u_rms: float = 0.04, epochs: int = 20, batch: int = 4096, lr: float = 1e-3,
        eval_every: int = 250, kmax: int = 16, target_clip: float = 50.0, verbose: bool = True) -> dict:
    """The whole experiment (module docstring); returns the results dict."""
    import torch

    import lbm
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    sptr = stream.cuda_stream
    nc = fine // factor
    tau_c = 0.5 + (tau_f - 0.5) / factor
    steps_c = snapshots * every // factor
    log = (lambda *a: print(*a, flush=True)) if verbose else (lambda *a: None)

    # 1. initial field and the fine lattice
    u = hit_velocity(fine, seed, u_rms)
    uh = u.permute(1, 2, 3, 0).reshape(-1, 3).contiguous().cpu().numpy()
    del u
    torch.cuda.empty_cache()
    d = lbm.default_desc(nx=fine, ny=fine, nz=fine, mode=lbm.MODE_PHYSICS, precision=lbm.PREC_F32,
                         collision=lbm.COLL_BGK, tau=tau_f, periodic=(1, 1, 1))
    lat = lbm.Lattice(d)
    lat.set_stream(sptr)
    lat.init_from_moments(np.ones(fine ** 3, np.float32), uh)
    del uh
    d_rho, d_u = lat.device_moments()
    filt = torch.empty((10, nc ** 3), device="cuda")
    lbm.box_filter(d_rho, d_u, (fine,) * 3, factor, filt.data_ptr(), sptr)
    torch.cuda.synchronize()
    filt0 = filt.cpu().numpy()
    fine_spectra = {0: spectrum(filt[1:4].reshape(3, nc, nc, nc))}
    fine_ke = {0: float(0.5 * (filt[1:4].double() ** 2).sum(0).mean())}

    # 2. fine run, filtered snapshots, training samples
    m = samples_per_snapshot
    X = torch.empty((snapshots * m, lbm.CLOSURE_INPUTS), device="cuda")
    T = torch.empty(snapshots * m, device="cuda")
    W = torch.empty(snapshots * m, device="cuda")
    step_s = 0.0
    t_wall = _events()
    t_wall[0].record(stream)
    for s in range(snapshots):
        e0, e1 = _events()
        e0.record(stream)
        lat.step(every)
        e1.record(stream)
        lbm.box_filter(d_rho, d_u, (fine,) * 3, factor, filt.data_ptr(), sptr)
        lbm.closure_samples(filt.data_ptr(), (nc,) * 3, tau_c, cs0, 1000003 * (s + 1) + seed, m,
                            X[s * m].data_ptr(), T[s * m:].data_ptr(), W[s * m:].data_ptr(), sptr)
        step_c = (s + 1) * every // factor
        if ((s + 1) * every) % factor == 0 and step_c % eval_every == 0:
            fine_spectra[step_c] = spectrum(filt[1:4].reshape(3, nc, nc, nc))
            fine_ke[step_c] = float(0.5 * (filt[1:4].double() ** 2).sum(0).mean())
        e1.synchronize()
        step_s += e0.elapsed_time(e1) / 1e3
    t_wall[1].record(stream)
    lat.sync()
    torch.cuda.synchronize()
    fine_total_s = t_wall[0].elapsed_time(t_wall[1]) / 1e3
    lat.close()
    log(f"fine {fine}^3: {snapshots * every} steps, step time {step_s:.1f} s, with data {fine_total_s:.1f} s")

    # 3. training
    T.clamp_(-target_clip, target_clip)
    w64 = W.double()
    r_eff = float((w64 * T.double()).sum() / w64.sum())
    mean = X.double().mean(0).float().cpu().numpy()
    std = X.double().std(0).float().cpu().numpy()
    iscale = (1.0 / np.maximum(std, 1e-6)).astype(np.float32)
    tr = lbm.Trainer(init_net(seed, mean, iscale), lbm.adam_default(lr=lr))
    tr.set_stream(sptr)
    e0, e1 = _events()
    e0.record(stream)
    losses = tr.fit(X.data_ptr(), T.data_ptr(), W.data_ptr(), snapshots * m, batch, epochs, seed=seed)
    e1.record(stream)
    torch.cuda.synchronize()
    train_s = e0.elapsed_time(e1) / 1e3
    net = tr.net()
    tr.close()
    # network output over the dataset, for the record
    R = torch.empty(snapshots * m, device="cuda")
    lbm.closure_predict(net, X.data_ptr(), snapshots * m, R.data_ptr(), sptr)
    torch.cuda.synchronize()
    r_pred_w = float((w64 * R.double()).sum() / w64.sum())
    log(f"training: {epochs} epochs in {train_s:.2f} s, loss {losses[0]:.4g} -> {losses[-1]:.4g}; "
        f"weighted r*: data {r_eff:.3f}, network {r_pred_w:.3f}")
    del X, T, W, R

    # 4. coarse runs from the filtered initial field
    rho0 = np.ascontiguousarray(filt0[0])
    u0 = np.ascontiguousarray(filt0[1:4].T)
    runs = {"smagorinsky": _coarse_run(lbm, stream, nc, tau_c, cs0, rho0, u0, steps_c, eval_every),
            "learned": _coarse_run(lbm, stream, nc, tau_c, cs0, rho0, u0, steps_c, eval_every, net)}

    # 5. spectra errors against the filtered fine field
    res = {"fine": fine, "factor": factor, "coarse": nc, "tau_fine": tau_f, "tau_coarse": tau_c,
           "fine_steps": snapshots * every, "coarse_steps": steps_c, "cs0": cs0, "u_rms": u_rms,
           "samples": snapshots * m, "epochs": epochs, "batch": batch, "lr": lr,
           "train_s": train_s, "loss_first": float(losses[0]), "loss_last": float(losses[-1]),
           "r_weighted_data": r_eff, "r_weighted_net": r_pred_w,
           "fine_step_s": step_s, "fine_total_s": fine_total_s, "kmax": kmax}
    for name, r in runs.items():
        errs = {}
        for t, e in r["spectra"].items():
            ef = fine_spectra.get(t)
            if ef is None:
                continue
            k = np.arange(1, kmax + 1)
            errs[t] = np.abs(e[k] - ef[k]) / ef[k]
        final = max(errs) if errs else None
        res[name] = {
            "finite": r["finite"], "device_s": r["device_s"],
            "wall_ratio": step_s / r["device_s"] if r["device_s"] else None,
            "max_rel_err_final": float(errs[final].max()) if final else None,
            "mean_rel_err_final": float(errs[final].mean()) if final else None,
            "max_rel_err_all_times": float(max(v.max() for v in errs.values())) if errs else None,
            "mean_rel_err_all_times": float(np.mean([v.mean() for v in errs.values()])) if errs else None,
            "ke": {str(t): v for t, v in r["ke"].items()},
            "err_by_time": {str(t): [float(x) for x in v] for t, v in errs.items()},
        }
        log(f"{name}: finite {r['finite']}, {r['device_s']:.2f} s, max rel err k<={kmax} final "
            f"{res[name]['max_rel_err_final']}, all times {res[name]['max_rel_err_all_times']}")
    res["fine_ke"] = {str(t): v for t, v in fine_ke.items()}
    res["fine_spectrum_final"] = [float(x) for x in fine_spectra[max(fine_spectra)][: kmax + 1]]
    res["net"] = [float(x) for x in net]
    return res


def main(argv=None) -> int:
    import argparse
    import json
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    sub = ap.add_subparsers(dest="cmd", required=True)
    r = sub.add_parser("run")
    r.add_argument("--fine", type=int, default=512)
    r.add_argument("--factor", type=int, default=4)
    r.add_argument("--tau", type=float, default=0.508)
    r.add_argument("--snapshots", type=int, default=2000)
    r.add_argument("--every", type=int, default=8)
    r.add_argument("--samples", type=int, default=4096)
    r.add_argument("--cs", type=float, default=0.1)
    r.add_argument("--epochs", type=int, default=20)
    r.add_argument("--batch", type=int, default=4096)
    r.add_argument("--lr", type=float, default=1e-3)
    r.add_argument("--eval-every", type=int, default=250)
    r.add_argument("--seed", type=int, default=5)
    r.add_argument("--out", default=None, help="write the full results (with the network) here")
    a = ap.parse_args(argv)
    res = run(fine=a.fine, factor=a.factor, tau_f=a.tau, snapshots=a.snapshots, every=a.every,
              samples_per_snapshot=a.samples, cs0=a.cs, epochs=a.epochs, batch=a.batch, lr=a.lr,
              eval_every=a.eval_every, seed=a.seed)
    if a.out:
        with open(a.out, "w") as f:
            json.dump(res, f)
    brief = {k: v for k, v in res.items() if k not in ("net",)}
    for name in ("smagorinsky", "learned"):
        brief[name] = {k: v for k, v in res[name].items() if k not in ("err_by_time", "ke")}
    print(json.dumps(brief))
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
