"""Learned committor surrogate: a small CNN trained on pB labels produced by
this library's own shooting runs, used to screen grids before shooting.

* ``CommittorCNN``: the network of include/gasp.h (gasp_cnn_*): forward,
  gradients and Adam steps all run on the GPU (tcgen05 convolutions).
* ``harvest_snapshots``: grids snapshotted from a nucleation swarm while
  still between the basins.
* ``shoot``: pB (and the reference's bootstrap error) of each grid by
  committor shooting with compaction.
* ``screen``: surrogate prediction for every grid, shooting fallback for
  grids predicted near pB = 0.5.
"""
from __future__ import annotations

import ctypes as C
import time

import numpy as np

from . import _native as nat
from . import engine
from ._native import check, lib

NPARAM = 28097
_SHAPES = [(32, 9, 1), (32,), (32, 9, 32), (32,), (32, 9, 32), (32,), (32, 9, 32), (32,),
           (32,), (1,)]


def init_params(seed=0):
    """He-normal convolution weights, N(0, 0.1) head weights, zero biases."""
    rs = np.random.default_rng(seed)
    parts = []
    for i, shp in enumerate(_SHAPES):
        if len(shp) == 3:
            parts.append(rs.normal(0.0, np.sqrt(2.0 / (shp[1] * shp[2])), shp).ravel())
        elif i == 8:
            parts.append(rs.normal(0.0, 0.1, shp))
        else:
            parts.append(np.zeros(shp))
    out = np.concatenate(parts).astype(np.float32)
    assert out.size == NPARAM
    return out


class CommittorCNN:
    """Handle on a gasp_cnn_t (parameters, Adam state, activations on the GPU)."""

    def __init__(self, L=64, max_batch=1024, params=None, seed=0):
        assert lib().gasp_cnn_param_count() == NPARAM
        self.L, self.max_batch = int(L), int(max_batch)
        self._h = C.c_void_p()
        check(lib().gasp_cnn_create(self.L, self.max_batch, C.byref(self._h)), "gasp_cnn_create")
        self.set_params(init_params(seed) if params is None else params)

    def set_params(self, params):
        p = np.ascontiguousarray(params, np.float32)
        assert p.size == NPARAM
        check(lib().gasp_cnn_set_params(self._h, p), "gasp_cnn_set_params")

    def get_params(self):
        out = np.empty(NPARAM, np.float32)
        check(lib().gasp_cnn_get_params(self._h, out), "gasp_cnn_get_params")
        return out

    def _spins(self, grids):
        g = np.ascontiguousarray(grids, np.int8).reshape(-1, self.L, self.L)
        return g

    def predict(self, grids, with_mag=False):
        """pB estimates of int8 grids; with_mag=True also returns each grid's
        magnetisation, computed on the device from the same upload."""
        g = self._spins(grids)
        out = np.empty(g.shape[0], np.float32)
        mag = np.empty(g.shape[0], np.float32) if with_mag else None
        if g.shape[0]:
            # one call: chunks of max_batch, uploads overlapped with the network
            check(lib().gasp_cnn_predict_ex(self._h, g.reshape(-1), g.shape[0], out,
                                            mag.ctypes.data if with_mag else None),
                  "gasp_cnn_predict_ex")
        return (out, mag) if with_mag else out

    def gradients(self, grids, labels):
        g = self._spins(grids)
        y = np.ascontiguousarray(labels, np.float32)
        loss = C.c_float()
        grad = np.empty(NPARAM, np.float32)
        check(lib().gasp_cnn_gradients(self._h, g.reshape(-1), y, g.shape[0], C.byref(loss),
                                       grad), "gasp_cnn_gradients")
        return float(loss.value), grad

    def train_step(self, grids, labels, lr):
        g = self._spins(grids)
        y = np.ascontiguousarray(labels, np.float32)
        loss = C.c_float()
        check(lib().gasp_cnn_train_step(self._h, g.reshape(-1), y, g.shape[0], float(lr),
                                        C.byref(loss)), "gasp_cnn_train_step")
        return float(loss.value)

    def train(self, grids, labels, epochs=20, batch=256, lr=2e-3, seed=0, augment=True,
              val=None, log=None, focus=0.0):
        """Mini-batch Adam.  augment: the 8 square symmetries (the
        Hamiltonian's), which leave pB unchanged.  focus > 0: each epoch draws
        its grids (with replacement) with weights 1 + focus * 4 y (1 - y), so
        grids with pB near 0.5 are seen more often than committed ones."""
        g = self._spins(grids)
        y = np.asarray(labels, np.float32)
        rs = np.random.default_rng(seed)
        w = 1.0 + focus * 4.0 * y.astype(np.float64) * (1.0 - y)
        w /= w.sum()
        hist = []
        for ep in range(epochs):
            order = (rs.permutation(g.shape[0]) if focus <= 0.0 else
                     rs.choice(g.shape[0], size=g.shape[0], p=w))
            losses = []
            for i in range(0, g.shape[0] - batch + 1, batch):
                idx = order[i:i + batch]
                xb = g[idx]
                if augment:
                    xb = _augment(xb, rs)
                losses.append(self.train_step(xb, y[idx], lr))
            rec = {"epoch": ep, "loss": float(np.mean(losses)) if losses else float("nan")}
            if val is not None:
                rec["val_mae"] = float(np.mean(np.abs(self.predict(val[0]) - val[1])))
            hist.append(rec)
            if log:
                log(rec)
        return hist

    def close(self):
        if self._h:
            lib().gasp_cnn_free(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _augment(xb, rs):
    """Each grid of the batch under one of the 8 symmetries of the square
    (k quarter turns, then an optional flip), drawn per grid; the grids of
    each symmetry are transformed together.  Circular translations are not
    drawn: with circular padding and a global average pool the network's
    output does not depend on them."""
    out = np.empty_like(xb)
    sym = rs.integers(8, size=xb.shape[0])
    for s_ in range(8):
        idx = np.nonzero(sym == s_)[0]
        if idx.size == 0:
            continue
        x = np.rot90(xb[idx], s_ & 3, axes=(1, 2))
        if s_ >= 4:
            x = x[:, :, ::-1]
        out[idx] = x
    return out


def shoot(grids, shots, beta, h, up=0.9, dn=-0.93, cap=20000, check_int=10, seed=1,
          rng="mwc64x", max_replicas=1 << 19, stats=None):
    """pB of each grid from `shots` trajectories (compaction on), each run
    until it reaches a basin or `cap` sweeps; unresolved trajectories are
    left out of pB as in the reference (src/mc_gpu.cu:812-826).  Returns
    (pB float64[n], attempts, seconds); `stats` (a dict) receives the number
    of trajectories and of unresolved ones."""
    g = np.ascontiguousarray(grids, np.int32)
    n, L = g.shape[0], g.shape[1]
    per = max(1, max_replicas // shots)
    pb = np.empty(n)
    attempts, t0 = 0, time.perf_counter()
    for i in range(0, n, per):
        block = g[i:i + per]
        k = block.shape[0]
        dg = engine.DeviceGrids(L, k * shots)
        dg.upload_inputs(block)
        r = engine.RngStates(k * shots, seed + i, kind=rng)
        res, fates, _, att = engine.run_driver(dg, r, beta, h, cap, check_int, cap, itask=1,
                                               dn_thr=dn, up_thr=up, ninputs=k, compact=True)
        pb[i:i + k] = res
        attempts += att
        if stats is not None:
            stats["trajectories"] = stats.get("trajectories", 0) + k * shots
            stats["unresolved"] = stats.get("unresolved", 0) + int(np.count_nonzero(fates == -1))
        dg.close()
        r.close()
    return pb, attempts, time.perf_counter() - t0


def harvest_snapshots(n, L=64, beta=0.54, h=0.07, replicas=32768, tot=12000, every=10,
                      lo=-0.93, hi=-0.65, seed=3, rng="mwc64x", bins=14):
    """Grids from a nucleation swarm, taken every `every` sweeps while their
    magnetisation lies in (lo, hi), balanced over `bins` magnetisation bins so
    that the barrier region is not drowned by metastable states.  The default
    window spans the metastable edge (m just above the A threshold -0.93)
    to grids whose droplet is well past the critical size."""
    dg = engine.DeviceGrids(L, replicas, -np.ones((replicas, L, L), np.int32))
    r = engine.RngStates(replicas, seed, kind=rng)
    pool = [[] for _ in range(bins)]
    cap_per_bin = 4 * n // bins + 1
    edges = np.linspace(lo, hi, bins + 1)

    def take(L_, ng_, payload, isweep, mag):
        m = np.asarray(mag, np.float64)
        sel = np.nonzero((m > lo) & (m < hi))[0]
        if sel.size == 0:
            return 0
        which = np.clip(np.searchsorted(edges, m[sel]) - 1, 0, bins - 1)
        nb = L_ * L_ // 8  # bytes per grid (L*L is a multiple of 8 here)
        for b in range(bins):
            ids = sel[which == b]
            room = cap_per_bin - len(pool[b])
            if room > 0 and ids.size:
                for j in ids[:room]:
                    bits = np.unpackbits(payload[j * nb:(j + 1) * nb], bitorder="little")
                    pool[b].append(np.where(bits.reshape(L_, L_) == 1, 1, -1).astype(np.int8))
        return 0

    engine.run_driver(dg, r, beta, h, tot, every, every, itask=0, dn_thr=-0.95, up_thr=0.999,
                      packed_out=take)
    dg.close()
    r.close()
    rs = np.random.default_rng(seed)
    per_bin = max(1, n // bins)
    out = []
    for b in range(bins):
        items = pool[b]
        if items:
            idx = rs.permutation(len(items))[:per_bin]
            out.extend(items[i] for i in idx)
    rest = [x for b in range(bins) for x in pool[b]]
    while len(out) < n and rest:
        out.append(rest[int(rs.integers(len(rest)))])
    return np.stack(out[:n]) if out else np.zeros((0, L, L), np.int8)


def screen(cnn, grids, beta, h, fallback_shots=128, band=0.1, window=None, **shoot_kw):
    """Surrogate pB for every grid; grids predicted within `band` of 0.5, and
    (window=(lo, hi), the magnetisation range the network was trained on)
    grids whose magnetisation lies outside it, are shot instead.  Returns
    (pB, fallback mask, seconds)."""
    t0 = time.perf_counter()
    if window is None:
        pred = cnn.predict(grids).astype(np.float64)
        near = np.abs(pred - 0.5) < band
    else:
        pred, mag = cnn.predict(grids, with_mag=True)
        pred = pred.astype(np.float64)
        near = (np.abs(pred - 0.5) < band) | (mag <= window[0]) | (mag >= window[1])
    out = pred.copy()
    if near.any():
        pb, _, _ = shoot(np.asarray(grids)[near], fallback_shots, beta, h, **shoot_kw)
        out[near] = pb
    return out, near, time.perf_counter() - t0


def run_experiment(n_train=20000, train_shots=256, n_test=2000, test_shots=1024,
                   n_screen=100000, baseline_shots=64, epochs=120, batch=1024, lr=2e-3, beta=0.54,
                   h=0.07, seed=0, log=None, focus=3.0):
    """Train the surrogate on shooting labels and measure what it gains.

    Returns a dict with the held-out MAE (surrogate alone and screened with
    fallback) against `test_shots`-shot labels, the MAE of `baseline_shots`
    shooting on the same grids, and the configurations/s of screening vs
    shooting alone with `baseline_shots` (whose binomial MAE is about 0.05
    at pB = 0.5)."""
    t = {}
    t0 = time.perf_counter()
    snaps = harvest_snapshots(n_train + n_test + n_screen, beta=beta, h=h, seed=seed + 3)
    t["harvest_s"] = time.perf_counter() - t0
    rs = np.random.default_rng(seed)
    snaps = snaps[rs.permutation(snaps.shape[0])]
    tr, te, sc = (snaps[:n_train], snaps[n_train:n_train + n_test],
                  snaps[n_train + n_test:])
    y_tr, a_tr, s_tr = shoot(tr, train_shots, beta, h, seed=seed + 11)
    y_te, a_te, s_te = shoot(te, test_shots, beta, h, seed=seed + 13)
    t["label_train_s"], t["label_test_s"] = s_tr, s_te
    net = CommittorCNN(64, batch, init_params(seed))
    t0 = time.perf_counter()
    hist = net.train(tr, y_tr, epochs=epochs, batch=batch, lr=lr, seed=seed,
                     val=(te, y_te), log=log, focus=focus)
    t["train_s"] = time.perf_counter() - t0
    pred_te = net.predict(te).astype(np.float64)
    mae_surrogate = float(np.mean(np.abs(pred_te - y_te)))
    window = (-0.93, -0.65)  # the harvest window: the network's training distribution
    scr_te, near_te, _ = screen(net, te, beta, h, fallback_shots=baseline_shots, window=window,
                                seed=seed + 17)
    mae_screened = float(np.mean(np.abs(scr_te - y_te)))
    # the screening question: is pB in [0.3, 0.7]?
    want, got = (y_te >= 0.3) & (y_te <= 0.7), (scr_te >= 0.3) & (scr_te <= 0.7)
    tp = int(np.count_nonzero(want & got))
    base_te, _, _ = shoot(te, baseline_shots, beta, h, seed=seed + 19)
    mae_baseline = float(np.mean(np.abs(base_te - y_te)))
    # MAE of shooting alone with fewer shots on the same held-out grids
    mae_by_shots = {baseline_shots: mae_baseline}
    for k, ns in enumerate((8, 16, 32)):
        est, _, _ = shoot(te, ns, beta, h, seed=seed + 41 + k)
        mae_by_shots[ns] = float(np.mean(np.abs(est - y_te)))
    mid = (y_te >= 0.1) & (y_te <= 0.9)
    # throughput on the screening pool, at the reference committor cap (20000
    # sweeps) and at a short cap that bounds the slowest trajectories
    t0 = time.perf_counter()
    net.predict(sc)
    t_cnn = time.perf_counter() - t0
    arms = {}
    for cap in (20000,):
        # The screened arm's time is set by its slowest fallback trajectories,
        # so it is taken three times (fresh shooting seeds) and the median kept.
        st_fb, st_sh, t_scr = {}, {}, []
        for rep in range(3):
            _, near_sc, ts = screen(net, sc, beta, h, fallback_shots=baseline_shots,
                                    window=window, seed=seed + 23 + 101 * rep, cap=cap,
                                    stats=st_fb)
            t_scr.append(ts)
        t_scr_med = float(np.median(t_scr))
        _, a_sh, t_sh = shoot(sc, baseline_shots, beta, h, seed=seed + 29, cap=cap, stats=st_sh)
        arms[cap] = {"screen_s": t_scr_med, "screen_s_runs": t_scr, "shoot_s": t_sh,
                     "speedup": t_sh / t_scr_med,
                     "speedup_range": [t_sh / max(t_scr), t_sh / min(t_scr)],
                     "screen_grids_per_s": sc.shape[0] / t_scr_med,
                     "shoot_grids_per_s": sc.shape[0] / t_sh,
                     "fallback_unresolved": st_fb.get("unresolved", 0),
                     "shoot_unresolved": st_sh.get("unresolved", 0),
                     "shoot_attempts_per_s": a_sh / t_sh}
    t_screen, t_shoot = arms[20000]["screen_s"], arms[20000]["shoot_s"]
    # shooting alone with the fewest shots whose held-out MAE is at most the
    # screened pipeline's (equal accuracy; the largest tried if none is), and
    # with the fewest whose MAE is <= 0.05 (the bar)
    for name, target in (("equal_mae", mae_screened), ("bar_0.05", 0.05)):
        few = min((k for k, v in mae_by_shots.items() if v <= target), default=baseline_shots)
        if few == baseline_shots:
            t_few = t_shoot
        else:
            _, _, t_few = shoot(sc, few, beta, h, seed=seed + 31)
        arms[name] = {"shots": few, "mae": mae_by_shots[few], "target_mae": target,
                      "shoot_s": t_few, "shoot_grids_per_s": sc.shape[0] / t_few,
                      "speedup": t_few / t_screen}
    res = {
        "n_train": int(tr.shape[0]), "train_shots": train_shots, "n_test": int(te.shape[0]),
        "test_shots": test_shots, "n_screen": int(sc.shape[0]), "baseline_shots": baseline_shots,
        "mae_surrogate": mae_surrogate, "mae_screened": mae_screened,
        "mae_shooting_baseline": mae_baseline, "fallback_fraction": float(near_sc.mean()),
        "mae_shooting_by_shots": {str(k): v for k, v in sorted(mae_by_shots.items())},
        "test_mid_0.1_0.9": {"n": int(mid.sum()),
                             "mae_surrogate": float(np.mean(np.abs(pred_te[mid] - y_te[mid]))),
                             "mae_screened": float(np.mean(np.abs(scr_te[mid] - y_te[mid]))),
                             "mae_shooting_baseline": float(np.mean(np.abs(base_te[mid] -
                                                                          y_te[mid])))},
        "screen_grids_per_s": sc.shape[0] / t_screen, "shoot_grids_per_s": sc.shape[0] / t_shoot,
        "speedup": t_shoot / t_screen, "final_train_loss": hist[-1]["loss"],
        "by_cap": {str(k): v for k, v in arms.items()},
        "cnn_only_grids_per_s": sc.shape[0] / t_cnn,
        "label_hist_train": np.histogram(y_tr, bins=10, range=(0.0, 1.0))[0].tolist(),
        "label_hist_test": np.histogram(y_te, bins=10, range=(0.0, 1.0))[0].tolist(),
        "band_0.3_0.7": {"test_in_band": int(want.sum()), "flagged": int(got.sum()),
                         "true_positives": tp},
        "label_mean_train": float(y_tr.mean()), "times_s": t,
        "history": hist,
    }
    net.close()
    return res


__all__ = ["CommittorCNN", "init_params", "shoot", "harvest_snapshots", "screen",
           "run_experiment", "nat"]
