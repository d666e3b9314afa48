"""Learned sub-grid closure: decaying homogeneous isotropic turbulence (HIT),
the fine plain-LBM run that generates training data, the trainer and the
coarse runs it is evaluated on.

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


class FineRun:
    """A fine periodic plain-BGK HIT run and what the closure needs from it:
    the filtered initial field, filtered spectra and kinetic energy every
    `eval_every` coarse steps, and (collect=True) the training samples on the
    device."""

    def __init__(self, fine=512, factor=4, tau_f=0.508, snapshots=2000, every=8,
                 samples_per_snapshot=4096, cs0=0.1, seed=5, u_rms=0.04, eval_every=250,
                 collect=True, stream=None):
        import torch

        import lbm
        self.fine, self.factor, self.tau_f, self.seed = fine, factor, tau_f, seed
        self.nc = nc = fine // factor
        self.tau_c = 0.5 + (tau_f - 0.5) / factor
        self.steps_c = snapshots * every // factor
        self.eval_every = eval_every
        stream = stream or torch.cuda.current_stream()
        sptr = stream.cuda_stream
        u = hit_velocity(fine, seed, u_rms)
        uh = u.permute(1, 2, 3, 0).reshape(-1, 3).contiguous().cpu().numpy()
        del u
        torch.cuda.empty_cache()
        d = lbm.default_desc(nx=fine, ny=fine, nz=fine, mode=lbm.MODE_PHYSICS,
                             precision=lbm.PREC_F32, collision=lbm.COLL_BGK, tau=tau_f,
                             periodic=(1, 1, 1))
        lat = lbm.Lattice(d)
        lat.set_stream(sptr)
        lat.init_from_moments(np.ones(fine ** 3, np.float32), uh)
        del uh
        d_rho, d_u = lat.device_moments()
        filt = torch.empty((10, nc ** 3), device="cuda")
        lbm.box_filter(d_rho, d_u, (fine,) * 3, factor, filt.data_ptr(), sptr)
        torch.cuda.synchronize()
        self.filt0 = filt.cpu().numpy()
        self.spectra = {0: spectrum(filt[1:4].reshape(3, nc, nc, nc))}
        self.ke = {0: float(0.5 * (filt[1:4].double() ** 2).sum(0).mean())}
        m = samples_per_snapshot
        self.n_samples = snapshots * m if collect else 0
        if collect:
            self.X = torch.empty((snapshots * m, lbm.CLOSURE_INPUTS), device="cuda")
            self.T = torch.empty(snapshots * m, device="cuda")
            self.W = torch.empty(snapshots * m, device="cuda")
        self.step_s = 0.0
        t_wall = _events()
        t_wall[0].record(stream)
        for s in range(snapshots):
            e0, e1 = _events()
            e0.record(stream)
            lat.step(every)
            e1.record(stream)
            step_c = (s + 1) * every // factor
            want_spec = ((s + 1) * every) % factor == 0 and step_c % eval_every == 0
            if collect or want_spec:
                lbm.box_filter(d_rho, d_u, (fine,) * 3, factor, filt.data_ptr(), sptr)
            if collect:
                lbm.closure_samples(filt.data_ptr(), (nc,) * 3, self.tau_c, cs0,
                                    1000003 * (s + 1) + seed, m, self.X[s * m].data_ptr(),
                                    self.T[s * m:].data_ptr(), self.W[s * m:].data_ptr(), sptr)
            if want_spec:
                self.spectra[step_c] = spectrum(filt[1:4].reshape(3, nc, nc, nc))
                self.ke[step_c] = float(0.5 * (filt[1:4].double() ** 2).sum(0).mean())
            e1.synchronize()
            self.step_s += e0.elapsed_time(e1) / 1e3
        t_wall[1].record(stream)
        lat.sync()
        torch.cuda.synchronize()
        self.total_s = t_wall[0].elapsed_time(t_wall[1]) / 1e3
        lat.close()

    def free(self):
        for k in ("X", "T", "W"):
            if hasattr(self, k):
                delattr(self, k)


def train(fr: FineRun, epochs=20, batch=4096, lr=1e-3, seed=5, target_clip=50.0, stream=None):
    """Fits a network to the run's samples; returns (network, info)."""
    import torch

    import lbm
    stream = stream or torch.cuda.current_stream()
    X, T, W = fr.X, fr.T, fr.W
    T.clamp_(-target_clip, target_clip)
    w64 = W.double()
    r_data = float((w64 * T.double()).sum() / w64.sum())
    mean = X.double().mean(0).float().cpu().numpy()
    std = X.double().std(0).float().cpu().numpy()
    iscale = (1.0 / np.maximum(std, 1e-6)).astype(np.float32)
    tr = lbm.Trainer(init_net(seed, mean, iscale), lbm.adam_default(lr=lr))
    tr.set_stream(stream.cuda_stream)
    e0, e1 = _events()
    e0.record(stream)
    losses = tr.fit(X.data_ptr(), T.data_ptr(), W.data_ptr(), fr.n_samples, batch, epochs, seed=seed)
    e1.record(stream)
    torch.cuda.synchronize()
    train_s = e0.elapsed_time(e1) / 1e3
    net = tr.net()
    tr.close()
    R = torch.empty(fr.n_samples, device="cuda")
    lbm.closure_predict(net, X.data_ptr(), fr.n_samples, R.data_ptr(), stream.cuda_stream)
    torch.cuda.synchronize()
    r_net = float((w64 * R.double()).sum() / w64.sum())
    return net, {"epochs": epochs, "batch": batch, "lr": lr, "train_s": train_s,
                 "loss": [float(x) for x in losses], "r_weighted_data": r_data,
                 "r_weighted_net": r_net, "samples": fr.n_samples}


def constant_net(r: float, like: np.ndarray) -> np.ndarray:
    """A network whose output is the constant r (zero weights, b3 =
    softplus^-1(r)); the standardisation is copied from `like`."""
    import lbm
    w = np.zeros(lbm.CLOSURE_FLOATS, np.float32)
    w[lbm.CLOSURE_PARAMS - 1] = math.log(math.expm1(r))
    w[lbm.CLOSURE_PARAMS:] = like[lbm.CLOSURE_PARAMS:]
    return w


def apriori_loss(net: np.ndarray, fr: FineRun, stream=None) -> float:
    """Weighted mean squared error sum w (r(x) - r*)^2 / sum w of a network
    over a run's samples (the fused forward/backward kernel's loss)."""
    import torch

    import lbm
    stream = stream or torch.cuda.current_stream()
    wsum = float(fr.W.double().sum())
    tr = lbm.Trainer(net)
    tr.set_stream(stream.cuda_stream)
    _, loss = tr.grad(fr.X.data_ptr(), fr.T.data_ptr(), fr.W.data_ptr(), fr.n_samples, 1.0 / wsum)
    tr.close()
    return loss


def coarse_run(fr: FineRun, cs: float, net=None, stream=None, step_variant: int = 0):
    """Coarse periodic BGK-Smagorinsky run (constant `cs`, or the learned
    closure with Cs^2 = cs^2 r when `net` is given) from the run's filtered
    initial field; device seconds of the steps, spectra and kinetic energy
    every eval_every steps.  step_variant 8 evaluates the closure's hidden
    layer on the tensor cores (bf16 activations)."""
    import torch

    import lbm
    stream = stream or torch.cuda.current_stream()
    nc = fr.nc
    d = lbm.default_desc(nx=nc, ny=nc, nz=nc, mode=lbm.MODE_PHYSICS, precision=lbm.PREC_F32,
                         collision=lbm.COLL_BGK, tau=fr.tau_c, periodic=(1, 1, 1), smagorinsky_cs=cs)
    lat = lbm.Lattice(d)
    lat.set_stream(stream.cuda_stream)
    if net is not None:
        lat.set_closure(net)
        if step_variant:
            lat.set_step_variant(step_variant)
    lat.init_from_moments(np.ascontiguousarray(fr.filt0[0]), np.ascontiguousarray(fr.filt0[1:4].T))
    secs, spectra, ke, ok = 0.0, {}, {}, True
    for s in range(0, fr.steps_c, fr.eval_every):
        e0, e1 = _events()
        e0.record(stream)
        lat.step(fr.eval_every)
        e1.record(stream)
        try:
            lat.sync()
        except lbm.LbmError:
            ok = False
            break
        torch.cuda.synchronize()
        secs += e0.elapsed_time(e1) / 1e3
        _, u = lat.read_moments()
        spectra[s + fr.eval_every] = spectrum_np(u, nc)
        ke[s + fr.eval_every] = float(0.5 * np.mean(np.sum(u.astype(np.float64) ** 2, axis=1)))
    lat.close()
    return {"device_s": secs, "spectra": spectra, "ke": ke, "finite": ok}


def errors(run: dict, fr: FineRun, kmax: int = 16) -> dict:
    """Relative spectral errors |E_c(k) - E_f(k)| / E_f(k), 1 <= k <= kmax,
    against the filtered fine run at matching times: at the last time
    (max and mean over k) and averaged over all times."""
    k = np.arange(1, kmax + 1)
    errs = {t: np.abs(e[k] - fr.spectra[t][k]) / fr.spectra[t][k]
            for t, e in run["spectra"].items() if t in fr.spectra}
    if not run["finite"] or not errs:
        return {"finite": False}
    last = max(errs)
    return {"finite": True, "device_s": run["device_s"],
            "final_max": float(errs[last].max()), "final_mean": float(errs[last].mean()),
            "time_mean": float(np.mean([v.mean() for v in errs.values()])),
            "time_max": float(max(v.max() for v in errs.values())),
            "ke_ratio": {str(t): run["ke"][t] / fr.ke[t] for t in run["ke"] if t in fr.ke},
            "by_time": {str(t): [float(x) for x in v] for t, v in errs.items()}}


def run(fine: int = 512, factor: int = 4, tau_f: float = 0.508, snapshots: int = 2000,
        every: int = 8, samples_per_snapshot: int = 4096, cs0: float = 0.1, seed: int = 5,
        u_rms: float = 0.04, epochs: int = 20, batch: int = 4096, lr: float = 1e-3,
        eval_every: int = 250, kmax: int = 16,
        calibrate=(0.1, 0.15, 0.2, 0.25, 0.35, 0.5, 0.75, 1.0, 1.5, 2.0), verbose: bool = True,
        tensor_cores: bool = False) -> dict:
    """The experiment: a training run (seed) gives the samples and, by a
    sweep of a single scale on Cs0 against its own filtered spectra, the
    calibration of the learned closure; a held-out run (seed + 1) is the
    evaluation: Smagorinsky Cs0 and the learned closure from its filtered
    initial field, compared with its filtered spectra."""
    import torch
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    log = (lambda *a: print(*a, flush=True)) if verbose else (lambda *a: None)
    variant = 8 if tensor_cores else 0  # step variant of the learned-closure coarse runs
    common = dict(fine=fine, factor=factor, tau_f=tau_f, snapshots=snapshots, every=every,
                  samples_per_snapshot=samples_per_snapshot, cs0=cs0, u_rms=u_rms,
                  eval_every=eval_every, stream=stream)
    tr_run = FineRun(seed=seed, collect=True, **common)
    log(f"training run {fine}^3 seed {seed}: {snapshots * every} steps in {tr_run.step_s:.1f} s")
    net, info = train(tr_run, epochs=epochs, batch=batch, lr=lr, seed=seed, stream=stream)
    r_const = info["r_weighted_data"]
    info["apriori_train"] = {"network": apriori_loss(net, tr_run, stream),
                             "best_constant": apriori_loss(constant_net(r_const, net), tr_run, stream),
                             "smagorinsky": apriori_loss(constant_net(1.0, net), tr_run, stream)}
    tr_run.free()
    log(f"training: {info['train_s']:.2f} s, loss {info['loss'][0]:.4g} -> {info['loss'][-1]:.4g}, "
        f"weighted r: data {info['r_weighted_data']:.3f} network {info['r_weighted_net']:.3f}")
    # calibration on the training run: one scale s on Cs0 (Cs^2 = s^2 cs0^2 r)
    cal = {}
    for a in calibrate:
        e = errors(coarse_run(tr_run, cs0 * math.sqrt(a), net, stream, variant), tr_run, kmax)
        cal[a] = e
        log(f"  calibration alpha {a}: time-mean err {e.get('time_mean')}")
    best = min((a for a in cal if cal[a]["finite"]), key=lambda a: cal[a]["time_mean"])
    # the same one-scale calibration of plain Smagorinsky, for comparison
    cal_s = {}
    for a in calibrate:
        cal_s[a] = errors(coarse_run(tr_run, cs0 * math.sqrt(a), None, stream), tr_run, kmax)
        log(f"  Smagorinsky alpha {a}: time-mean err {cal_s[a].get('time_mean')}")
    best_s = min((a for a in cal_s if cal_s[a]["finite"]), key=lambda a: cal_s[a]["time_mean"])
    ev_run = FineRun(seed=seed + 1, collect=True, **common)
    log(f"evaluation run seed {seed + 1}: {ev_run.step_s:.1f} s")
    ev_run.T.clamp_(-50.0, 50.0)
    info["apriori_heldout"] = {"network": apriori_loss(net, ev_run, stream),
                               "best_constant": apriori_loss(constant_net(r_const, net), ev_run, stream),
                               "smagorinsky": apriori_loss(constant_net(1.0, net), ev_run, stream)}
    log(f"a-priori weighted MSE on the held-out run: {info['apriori_heldout']}")
    ev_run.free()
    res = {"fine": fine, "factor": factor, "coarse": ev_run.nc, "tau_fine": tau_f,
           "tau_coarse": ev_run.tau_c, "fine_steps": snapshots * every, "coarse_steps": ev_run.steps_c,
           "cs0": cs0, "u_rms": u_rms, "kmax": kmax, "train_seed": seed, "eval_seed": seed + 1,
           "training": info, "calibration": {str(a): {k: v for k, v in e.items() if k != "by_time"}
                                              for a, e in cal.items()},
           "calibration_smagorinsky": {str(a): {k: v for k, v in e.items() if k != "by_time"}
                                        for a, e in cal_s.items()},
           "alpha": best, "alpha_smagorinsky": best_s, "fine_step_s": ev_run.step_s, "fine_total_s": ev_run.total_s,
           "fine_ke": {str(t): v for t, v in ev_run.ke.items()},
           "fine_spectrum_final": [float(x) for x in ev_run.spectra[max(ev_run.spectra)][: kmax + 1]],
           "net": [float(x) for x in net]}
    for name, cs, nn in (("smagorinsky", cs0, None), ("learned", cs0 * math.sqrt(best), net),
                         ("learned_uncalibrated", cs0, net),
                         ("smagorinsky_calibrated", cs0 * math.sqrt(best_s), None)):
        e = errors(coarse_run(ev_run, cs, nn, stream, variant if nn is not None else 0), ev_run, kmax)
        if e.get("device_s"):
            e["wall_ratio"] = ev_run.step_s / e["device_s"]
        res[name] = e
        log(f"{name}: final max {e.get('final_max')}, final mean {e.get('final_mean')}, "
            f"time mean {e.get('time_mean')}, wall ratio {e.get('wall_ratio')}")
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
    r.add_argument("--tensor-cores", action="store_true",
                   help="learned-closure coarse runs with the hidden layer on the tensor cores")
    a = ap.parse_args(argv)
    res = run(fine=a.fine, factor=a.factor, tau_f=a.tau, snapshots=a.snapshots, every=a.every,
              samples_per_snapshot=a.samples, cs0=a.cs, epochs=a.epochs, batch=a.batch, lr=a.lr,
              eval_every=a.eval_every, seed=a.seed, tensor_cores=a.tensor_cores)
    if a.out:
        with open(a.out, "w") as f:
            json.dump(res, f)
    brief = {k: v for k, v in res.items() if k not in ("net", "calibration", "calibration_smagorinsky")}
    for name in ("smagorinsky", "learned", "learned_uncalibrated", "smagorinsky_calibrated"):
        brief[name] = {k: v for k, v in res[name].items() if k not in ("by_time", "ke_ratio")}
    brief["training"] = {k: v for k, v in res["training"].items() if k != "loss"}
    print(json.dumps(brief))
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
