"""Parameter builders for the jet workloads.

``reference_like`` reproduces the reference's constexpr derivation from
(u, diam, Re, We, W) (src/constants.cuh:70-101,
src/functions/globalFunctions.cuh:68-104, 232-283) and its two-jet crossflow
boundary set; ``oil_jet`` states the configuration directly in lattice units
(tau, sigma, interface width, mobility, nozzle diameter, inlet speed and
noise), with exact periodic x and y faces and the oil inflow / outflow pair on z.
"""
from __future__ import annotations

import numpy as np

from . import _lib
from ._lib import Params

CS2_PHASE = np.float32(0.25)  # D3Q7 lattice sound speed squared (D3Q7.cuh:45-48)


def reference_like(nx, ny, nz, velocity_set=19, **kw) -> Params:
    """Reference derivation; keyword arguments as _lib.reference_params."""
    return _lib.reference_params(nx, ny, nz, velocity_set, **kw)


def oil_jet(nx, ny, nz, velocity_set=19, tau=0.55, sigma=1e-3, width=4.0, mobility=0.1, diam=8,
            w_in=0.05, noise=0.01, seed=0, storage=_lib.STORAGE_F32, periodic="exact",
            centre=None) -> Params:
    """Oil jet from a circular nozzle on the z = 0 face into quiescent water.

    tau is the hydrodynamic relaxation time of both phases (nu = (tau - 1/2)/3),
    mobility M sets the phase-field rate omega_g = 1/(1/2 + M/cs2) and the
    sharpening gamma = 4 M / (W cs2); the inlet speed per cell and step is
    w_in (1 + noise N(0, 1)) from the counter-based generator keyed by seed.
    periodic = "exact" wraps x and y; "copy" uses the reference's ghost-layer
    copy rule on both.
    """
    f32 = np.float32
    p = Params()
    p.nx, p.ny, p.nz = nx, ny, nz
    p.velocity_set = velocity_set
    p.storage = storage
    bc = _lib.BC_PERIODIC if periodic == "exact" else _lib.BC_PERIODIC_COPY
    p.bc_x = bc
    p.bc_y = bc
    p.bc_z = _lib.BC_JET
    nu = f32((tau - 0.5) / 3.0)
    p.nu_water = nu
    p.nu_oil = nu
    om = f32(1.0 / (0.5 + 3.0 * float(nu)))
    p.omco_water = f32(1.0) - om
    p.omco_oil = f32(1.0) - om
    p.omco_ref = f32(1.0) - om
    p.sigma = f32(sigma)
    p.gamma = f32(4.0 * mobility / (width * float(CS2_PHASE)))
    p.omega_g = f32(1.0 / (0.5 + mobility / float(CS2_PHASE)))
    cx, cy = centre if centre is not None else ((nx - 1) * 0.5, (ny - 1) * 0.5)
    r = int(diam) // 2
    p.oil_cx, p.oil_cy, p.oil_r2 = f32(cx), f32(cy), f32(r * r)
    p.u_oil = f32(w_in)
    p.water_cx, p.water_cz, p.water_r2 = f32(0), f32(0), f32(-1.0)  # no water disc
    p.u_water = f32(0)
    p.noise_amp = f32(noise)
    p.seed = int(seed)
    p.u_limit = f32(0.3)
    p.tile_z = 0
    return p


def periodic_box(n=(32, 32, 32), velocity_set=19, tau=0.6, sigma=1e-2, width=4.0, mobility=0.1,
                 storage=_lib.STORAGE_F32) -> Params:
    """Closed, fully periodic box (no inflow): the setting in which total phi
    and mass are exact invariants."""
    p = oil_jet(n[0], n[1], n[2], velocity_set, tau=tau, sigma=sigma, width=width, mobility=mobility,
                w_in=0.0, noise=0.0, storage=storage)
    p.bc_z = _lib.BC_PERIODIC
    p.oil_r2 = np.float32(-1.0)
    return p
