"""Tracer pieces that need no GPU: the Philox4x32-10 restatement against the
published known-answer vectors of the Random123 distribution (Salmon et al.
2011), seeding (reference particles_init_mode, plane quotas, plane ids), the
Dm ladder's crossed design (README "Per-particle diffusivities"), and the
statistics of the oracle's random walk (mean-square displacement 2 Dm t per
axis; no z motion in 2-D, README "2D runs")."""
import numpy as np

from felbm_gpu_b200 import geometry
from felbm_gpu_b200.tracers import dm_ladder, seed
from oracle import tracers_ref as tr


def test_philox_known_answers():
    kat = [((0, 0, 0, 0), (0, 0), (0x6627e8d5, 0xe169c58d, 0xbc57ac4c, 0x9b00dbd8)),
           ((0xffffffff,) * 4, (0xffffffff,) * 2, (0x408f276d, 0x41c83b0e, 0xa20bc7c6, 0x6d5451fd)),
           ((0x243f6a88, 0x85a308d3, 0x13198a2e, 0x03707344), (0xa4093822, 0x299f31d0),
            (0xd16cfe09, 0x94fdcceb, 0x5001e420, 0x24126ea1))]
    for c, k, want in kat:
        got = tr.philox4x32_10(*[np.array([x]) for x in c], *k)
        assert tuple(int(v[0]) for v in got) == want


def test_normals_are_standard():
    ids = np.arange(200000)
    z0, z1 = tr.normal_pair(7, ids, 3, 0, 0)
    for z in (z0, z1):
        assert abs(z.mean()) < 0.01 and abs(z.std() - 1.0) < 0.01
    assert abs(np.corrcoef(z0, z1)[0, 1]) < 0.01


def test_plane_seeding_quota_and_fluid():
    solid = geometry.spheres((16, 24, 32), 3.0, 10, 3.0, 5)
    pos, pid = seed(solid, 500, mode="plane", axis=0, offsets=(4.0, 20.0), rng_seed=3)
    assert pos.shape == (3, 1000) and np.array_equal(np.bincount(pid), [500, 500])
    assert np.all(pos[0, pid == 0] == 4.0) and np.all(pos[0, pid == 1] == 20.0)
    nz, ny, nx = solid.shape
    ix = np.floor(pos + 0.5).astype(int) % np.array([[nx], [ny], [nz]])
    assert not solid[ix[2], ix[1], ix[0]].any()
    pos2, _ = seed(solid, 500, mode="plane", axis=0, offsets=(4.0, 20.0), rng_seed=3)
    assert np.array_equal(pos, pos2)


def test_volume_seeding_2d_has_z_zero():
    solid, _ = geometry.cylinders((1, 40, 40), 3.0, 6.0, 0.6, seed=1)
    pos, pid = seed(solid, 300, rng_seed=1)
    assert np.all(pos[2] == 0.0) and np.all(pid == 0)


def test_dm_ladder_crossed_design():
    pid = np.repeat([0, 1], 6)
    dm = dm_ladder([(1e-3, 2), (1e-2, 4)], pid)
    assert np.array_equal(dm[:6], [1e-3, 1e-3, 1e-2, 1e-2, 1e-2, 1e-2])
    assert np.array_equal(dm[6:], dm[:6])


def test_oracle_random_walk_statistics():
    """No flow, all fluid: after t steps each axis has variance 2 Dm t (95 %
    interval of the sample variance of n normals: +-2.8 sqrt(2/n))."""
    shape = (32, 32, 32)
    solid = np.zeros(shape, np.uint8)
    u = np.zeros((3, 32 ** 3))
    n, dm, steps = 20000, 0.05, 40
    pos = np.full((3, n), 16.0)
    ids = np.arange(n)
    for t in range(steps):
        pos, _ = tr.step(pos, np.full(n, dm), ids, u, solid, t, substeps=2, order=2, seed=11)
    var = ((pos - 16.0) ** 2).mean(axis=1)
    want = 2 * dm * steps
    assert np.all(np.abs(var / want - 1.0) < 2.8 * np.sqrt(2.0 / n)), var / want


def test_oracle_2d_no_z_kick():
    solid = np.zeros((1, 16, 16), np.uint8)
    u = np.zeros((3, 256))
    pos = np.stack([np.full(50, 8.0), np.full(50, 8.0), np.zeros(50)])
    for t in range(5):
        pos, _ = tr.step(pos, np.full(50, 0.1), np.arange(50), u, solid, t)
    assert np.all(pos[2] == 0.0) and np.std(pos[0]) > 0


def _fluid_box(nx=40, ny=40, nz=8):
    return np.zeros((nz, ny, nx), np.uint8)


def _linear_field(solid, fn):
    nz, ny, nx = solid.shape
    z, y, x = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    ux, uy, uz = fn(x.astype(float), y.astype(float), z.astype(float))
    return np.stack([np.broadcast_to(a, solid.shape).reshape(-1) for a in (ux, uy, uz)]).astype(np.float64)


def test_stretching_uniform_shear_is_exact():
    """u = (g y, 0, 0): J is nilpotent, so the Euler update of the line
    element is exact and log|rho| = log|rho0 + t J rho0| (reference analytic
    test, docs/HANDOFF_stretching.md section 3.3: shear error ~4e-15)."""
    solid = _fluid_box()
    gam = 0.01
    u = _linear_field(solid, lambda x, y, z: (gam * y, 0 * y, 0 * y))
    n = 64
    rng = np.random.default_rng(1)
    pos = np.stack([rng.uniform(5, 10, n), rng.uniform(8, 30, n), rng.uniform(2, 5, n)])
    ids = np.arange(n)
    rh0 = tr.orientations(ids, 5)
    rh, lr = rh0.copy(), np.zeros(n)
    steps, subs = 20, 3
    for s in range(steps):
        pos, _, rh, lr, row = tr.step(pos, np.zeros(n), ids, u, solid, s, substeps=subs, order=1, stretch=(rh, lr))
    J = np.array([[0, gam, 0], [0, 0, 0], [0, 0, 0]])
    want = np.log(np.linalg.norm(rh0 + steps * (J @ rh0), axis=0))
    assert np.max(np.abs(lr - want)) < 1e-13, np.max(np.abs(lr - want))
    assert np.max(np.abs(np.linalg.norm(rh, axis=0) - 1.0)) < 1e-14
    assert row[0] == steps and row[4] == n
    # Eq. (12) of the last step: mean of gamma rho_x rho_y over tracers and substeps
    assert np.isfinite(row[1]) and np.isnan(row[5]) and np.isnan(row[6])


def test_stretching_rotation_has_zero_lambda():
    """Solid-body rotation: J antisymmetric, so Eq. (12) is zero to rounding
    while explicit Euler inflates |rho| (the reference's rotation case)."""
    solid = _fluid_box()
    om = 0.02
    u = _linear_field(solid, lambda x, y, z: (-om * (y - 20), om * (x - 20), 0 * z))
    n = 50
    rng = np.random.default_rng(2)
    pos = np.stack([rng.uniform(17, 23, n), rng.uniform(17, 23, n), rng.uniform(2, 5, n)])
    ids = np.arange(n)
    rh, lr = tr.orientations(ids, 9), np.zeros(n)
    for s in range(10):
        pos, _, rh, lr, row = tr.step(pos, np.zeros(n), ids, u, solid, s, substeps=2, order=2, stretch=(rh, lr))
        assert abs(row[1]) < 1e-16
    assert np.all(lr > 0) and np.max(lr) < 10 * 2 * 0.5 * np.log1p((om * 0.5) ** 2) + 1e-15


def test_stretching_phase_split_recombines():
    """n_w + n_nw = n_active and (n_w lambda_w + n_nw lambda_nw) / n_active =
    lambda (reference checks, docs/HANDOFF_stretching.md section 4)."""
    solid = geometry.spheres((12, 30, 30), 2.5, 6, 2.0, 3)
    nz, ny, nx = solid.shape
    u = _linear_field(solid, lambda x, y, z: (0.01 * np.sin(y / 5.0), 0.004 * np.cos(x / 4.0), 0.002 * np.sin(z)))
    u[:, solid.reshape(-1) != 0] = 0.0
    cg = _linear_field(solid, lambda x, y, z: (0.5 + 0.5 * np.sin(x / 3.0), 0 * x, 0 * x))[0]
    pos, _ = seed(solid, 300, rng_seed=4)
    ids = np.arange(300)
    rh, lr = tr.orientations(ids, 1), np.zeros(300)
    for s in range(6):
        pos, _, rh, lr, row = tr.step(pos, np.full(300, 1e-3), ids, u, solid, s, substeps=2, stretch=(rh, lr),
                                      cgrid=cg)
        assert row[7] + row[8] == row[4]
        assert abs((row[7] * row[5] + row[8] * row[6]) / row[4] - row[1]) < 1e-14
