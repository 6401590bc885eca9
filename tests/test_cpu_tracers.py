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
