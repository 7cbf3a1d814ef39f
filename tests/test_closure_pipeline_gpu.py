"""End-to-end learned closure at small scale: the solver's own fine run
produces the training data, the network trains on the GPU, and the trained
closure beats the method without it on a held-out snapshot."""
import numpy as np
import pytest

from ssmdlbm_b200 import configs


@pytest.mark.gpu
def test_closure_experiment_small():
    from ssmdlbm_b200 import closure
    fine = configs.oil_jet(32, 32, 128, 19, tau=0.55, sigma=1e-3, mobility=0.1, diam=8, w_in=0.05, noise=0.01,
                           seed=0)
    r = closure.experiment(fine, steps=1200, sample_every=100, spinup=400, train_steps=300, batch=16384,
                           lr=2e-3, seed=0, update_every=2)
    h = r["heldout_loss"]
    print("held-out loss", h, "errors plain", r["errors_plain"], "closure", r["errors_closure"])
    assert r["mlp_status"] == 0
    # what the trained network gains over the method without it (nu_t = 0, factor 1)
    assert h["trained"] < 0.5 * h["no_closure"], h
    assert h["trained"] < h["untrained"], h
    # both coarse runs are stable and the closure changes the flow
    assert np.all(np.isfinite(r["closure"].centreline_uz))
    assert not np.array_equal(r["closure"].centreline_uz, r["plain"].centreline_uz)
    assert r["samples"] == 9 * 16 * 16 * 64


def test_coarse_params_scaling():
    from ssmdlbm_b200 import closure
    p = configs.oil_jet(64, 64, 256, 19, tau=0.55, sigma=1e-3, mobility=0.1, diam=8, w_in=0.05)
    q = closure.coarse_params(p)
    assert (q.nx, q.ny, q.nz) == (32, 32, 128)
    assert q.nu_water == np.float32(p.nu_water) * np.float32(0.5)
    assert abs(q.sigma - p.sigma / 2) < 1e-12 and q.gamma == p.gamma  # the interface keeps its physical width
    assert abs(q.oil_r2 - p.oil_r2 / 4) < 1e-6 and abs(q.oil_cx - 15.5) < 1e-6
    mob_f = (1 / p.omega_g - 0.5) * 0.25
    mob_c = (1 / q.omega_g - 0.5) * 0.25
    assert abs(mob_c - mob_f / 2) < 1e-6
    assert q.u_oil == p.u_oil and q.closure is None


def test_fine_centreline_covers_the_coarse_sample():
    """The fine run's centreline is averaged over the fine cells under the
    coarse cells the coarse run samples (fine 2i, 2i + 1 under coarse i)."""
    from ssmdlbm_b200 import closure
    assert closure._coarse_axis_cells(31.5) == [31, 32]  # centred nozzle, even coarse size
    assert closure._coarse_axis_cells(15.0) == [15]      # a nozzle on a cell centre
    p = configs.oil_jet(128, 96, 256, 19, diam=16)
    q = closure.coarse_params(p)
    xs = [2 * i + 0.5 for i in closure._coarse_axis_cells(float(q.oil_cx))]
    ys = [2 * j + 0.5 for j in closure._coarse_axis_cells(float(q.oil_cy))]
    # the 2 x 2 fine blocks tile a 4 x 4 patch centred on the fine nozzle axis
    assert xs == [62.5, 64.5] and abs(np.mean(xs) - float(p.oil_cx)) < 1e-6
    assert ys == [46.5, 48.5] and abs(np.mean(ys) - float(p.oil_cy)) < 1e-6
