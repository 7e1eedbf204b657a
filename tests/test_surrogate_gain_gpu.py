"""What the trained committor surrogate gains over shooting alone, end to end
on a B200 at a small scale: droplet grids of the committor workload's kind
(L=64, all -1 with a centred +1 disc of radius U[4,12], 2 % of sites
flipped), training labels from 32-shot shooting, held-out labels from
256-shot shooting, a network trained on the GPU, then screening (network for
every grid, 64-shot shooting for grids predicted within 0.1 of 0.5) against
shooting every grid with 64 trajectories.  The gain is measured as attempted
flips, which do not depend on host timing, and as wall time of the whole
screening (network included) against shooting alone."""
import numpy as np
import pytest

from gpu_2dising_b200 import engine, surrogate

pytestmark = pytest.mark.gpu

L, BETA, H = 64, 0.54, 0.07


@pytest.fixture(scope="module", autouse=True)
def device():
    return engine.init_device(0)


def _droplets(n, seed):
    rs = np.random.default_rng(seed)
    yy, xx = np.mgrid[0:L, 0:L]
    d2 = (yy - L / 2) ** 2 + (xx - L / 2) ** 2
    r = rs.uniform(4.0, 12.0, size=n)
    g = np.where(d2[None] <= (r * r)[:, None, None], 1, -1).astype(np.int8)
    flip = rs.random((n, L, L)) < 0.02
    g[flip] = -g[flip]
    return g


def test_trained_surrogate_gains_over_shooting_alone():
    train, test, cands = _droplets(1536, 11), _droplets(256, 12), _droplets(2048, 13)
    y_train, _, _ = surrogate.shoot(train, 32, BETA, H, seed=21)
    y_test, _, _ = surrogate.shoot(test, 256, BETA, H, seed=22)
    assert 0.05 < float(np.mean(y_train)) < 0.95  # both basins are represented

    net = surrogate.CommittorCNN(L, 256, surrogate.init_params(5))
    mae_untrained = float(np.mean(np.abs(net.predict(test) - y_test)))
    net.train(train, y_train.astype(np.float32), epochs=24, batch=256, lr=3e-3, seed=3, focus=3.0)
    mae_net = float(np.mean(np.abs(net.predict(test) - y_test)))
    pb_scr, near_test, _ = surrogate.screen(net, test, BETA, H, fallback_shots=64, band=0.1,
                                            seed=23)
    mae_screened = float(np.mean(np.abs(pb_scr - y_test)))

    # screening the candidates: network for all, shooting for the flagged ones
    pred = net.predict(cands).astype(np.float64)
    near = np.abs(pred - 0.5) < 0.1
    st_fb, st_all = {}, {}
    _, att_fallback, t_fallback = surrogate.shoot(cands[near], 64, BETA, H, seed=24, stats=st_fb)
    # the method without the network: every candidate shot 64 times
    _, att_all, t_all = surrogate.shoot(cands, 64, BETA, H, seed=24, stats=st_all)
    gain = att_all / max(att_fallback, 1)
    # wall time of the whole screening, the network's prediction included; the
    # best of repeated runs on both sides, so that a one-off host stall (an
    # allocation, another process) does not decide the ratio
    t_all = min(t_all, surrogate.shoot(cands, 64, BETA, H, seed=25)[2])
    t_screen = np.inf
    for rep in range(3):
        _, near_s, ts = surrogate.screen(net, cands, BETA, H, fallback_shots=64, band=0.1,
                                         seed=24 + rep)
        t_screen = min(t_screen, ts)
    time_gain = t_all / t_screen
    mid = (y_test >= 0.1) & (y_test <= 0.9)
    mae_mid = float(np.mean(np.abs(pb_scr[mid] - y_test[mid]))) if mid.any() else 0.0
    print(f"MAE untrained {mae_untrained:.3f} trained {mae_net:.3f} screened {mae_screened:.3f} "
          f"(0.1<=pB<=0.9: {mae_mid:.3f}, {int(mid.sum())} grids); flagged {near.mean():.3f} of "
          f"candidates; attempts {att_all:.3e} vs {att_fallback:.3e} ({gain:.1f}x); time "
          f"{t_all:.2f} s shooting all vs {t_screen:.2f} s screening ({time_gain:.1f}x)")

    assert mae_net < 0.5 * mae_untrained
    assert mae_screened <= 0.05, mae_screened  # the per-grid accuracy bar
    assert mae_mid <= 0.08, mae_mid  # where shooting matters most (a small, noisy sample here)
    assert st_all["unresolved"] == 0 and st_fb.get("unresolved", 0) == 0
    assert near.mean() < 0.5
    # (the screening's own flags may differ from `near` at the band's edge: the
    # pooled sums are float atomics, so the last bit of a prediction can vary)
    assert abs(float(near_s.mean()) - float(near.mean())) < 0.01
    # on a B200: MAE 0.338 untrained, 0.030 trained, 0.028 screened; 9.1 % of the
    # candidates flagged; 10.9x fewer attempted flips, 2.5x less wall time.  At this
    # scale (2048 candidates) each shooting run has a latency floor set by its slowest
    # trajectories, so the wall-time gain stays below the attempts gain; at 100 000
    # candidates (bench.py --workload surrogate) it is ~25x.
    assert gain >= 6.0, gain
    assert time_gain >= 2.0, time_gain
