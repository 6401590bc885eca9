"""CPU restatement of the GPU tracer step — TEST INFRASTRUCTURE ONLY.

numpy FP64, the same definitions as felbm_gpu_b200/csrc/tracers.cuh (the
reference's ParticleManager is in the absent felbm_local tree, so the
integrator is this library's definition, written down once for the kernel and
once here): trilinear interpolation of a node-indexed velocity snapshot with
periodic wrap, Euler or Heun substeps, Brownian kicks sqrt(2 Dm dt) N(0,1)
from Philox4x32-10 (Salmon et al. 2011) with counter (id, step, substep,
draw) and the seed as key, Box-Muller normals from 53-bit uniforms, no z kick
in 2-D (where tracers do not move along z at all), moves onto solid nodes
rejected; optional Lagrangian stretching (unit orientation rho_hat and
log_rho per tracer, lambda_s = rho_hat . J rho_hat per accepted substep with J
the gradient of the trilinear interpolant, Benettin renormalisation, the
step's row of the stretching time series).
"""
from __future__ import annotations

import numpy as np

_M0, _M1 = np.uint64(0xD2511F53), np.uint64(0xCD9E8D57)
_W0, _W1 = np.uint64(0x9E3779B9), np.uint64(0xBB67AE85)
_MASK = np.uint64(0xFFFFFFFF)


def philox4x32_10(c0, c1, c2, c3, k0, k1):
    """Philox4x32-10 on uint32 arrays (returned as uint64 arrays < 2^32)."""
    c = [np.asarray(x, np.uint64) & _MASK for x in (c0, c1, c2, c3)]
    k0 = np.uint64(k0) & _MASK
    k1 = np.uint64(k1) & _MASK
    for _ in range(10):
        p0 = c[0] * _M0
        p1 = c[2] * _M1
        hi0, lo0 = p0 >> np.uint64(32), p0 & _MASK
        hi1, lo1 = p1 >> np.uint64(32), p1 & _MASK
        c = [hi1 ^ c[1] ^ k0, lo1, hi0 ^ c[3] ^ k1, lo0]
        k0 = (k0 + _W0) & _MASK
        k1 = (k1 + _W1) & _MASK
    return c


def normal_pair(seed: int, ids: np.ndarray, step: int, sub: int, draw: int):
    ids = np.asarray(ids, np.int64).astype(np.uint64)
    n = len(ids)
    c = philox4x32_10(ids & _MASK, ids >> np.uint64(32), np.full(n, step, np.uint64),
                      np.full(n, sub * 2 + draw, np.uint64), seed & 0xFFFFFFFF, (seed >> 32) & 0xFFFFFFFF)
    inv53 = 1.0 / 9007199254740992.0
    u1 = (((c[0] >> np.uint64(5)) << np.uint64(26)) | (c[1] >> np.uint64(6))).astype(np.float64)
    u1 = (u1 + 1.0) * inv53
    u2 = (((c[2] >> np.uint64(5)) << np.uint64(26)) | (c[3] >> np.uint64(6))).astype(np.float64) * inv53
    r = np.sqrt(-2.0 * np.log(u1))
    return r * np.cos(2.0 * np.pi * u2), r * np.sin(2.0 * np.pi * u2)


def velocity_grid(shape, nodes: np.ndarray, ux, uy, uz) -> np.ndarray:
    """(3, nodes) snapshot from per-site velocity (reference order) and the
    sites' node indices; solid nodes hold 0."""
    nz, ny, nx = shape
    u = np.zeros((3, nx * ny * nz))
    for a, v in enumerate((ux, uy, uz)):
        u[a, nodes] = v
    return u


def _wrap(x, L):
    x = np.fmod(x, L)
    x = np.where(x < 0.0, x + L, x)
    return np.where(x >= L, x - L, x)


def interp(u, shape, x, y, z):
    nz, ny, nx = shape
    fx, fy, fz = np.floor(x), np.floor(y), np.floor(z)
    ax, ay, az = x - fx, y - fy, z - fz
    x0, y0, z0 = fx.astype(np.int64) % nx, fy.astype(np.int64) % ny, fz.astype(np.int64) % nz
    x1, y1, z1 = (x0 + 1) % nx, (y0 + 1) % ny, (z0 + 1) % nz
    sy, sz = nx, nx * ny
    idx = [x0 + y0 * sy + z0 * sz, x1 + y0 * sy + z0 * sz, x0 + y1 * sy + z0 * sz, x1 + y1 * sy + z0 * sz,
           x0 + y0 * sy + z1 * sz, x1 + y0 * sy + z1 * sz, x0 + y1 * sy + z1 * sz, x1 + y1 * sy + z1 * sz]
    w = [(1 - ax) * (1 - ay) * (1 - az), ax * (1 - ay) * (1 - az), (1 - ax) * ay * (1 - az), ax * ay * (1 - az),
         (1 - ax) * (1 - ay) * az, ax * (1 - ay) * az, (1 - ax) * ay * az, ax * ay * az]
    out = []
    for a in range(3):
        s = np.zeros_like(x)
        for q in range(8):
            s = s + w[q] * u[a][idx[q]]
        out.append(s)
    return out


def interp_grad(u, shape, x, y, z):
    """Velocity (3 arrays) and its gradient J[a][b] = d u_a / d x_b of the
    trilinear interpolant."""
    nz, ny, nx = shape
    fx, fy, fz = np.floor(x), np.floor(y), np.floor(z)
    ax, ay, az = x - fx, y - fy, z - fz
    x0, y0, z0 = fx.astype(np.int64) % nx, fy.astype(np.int64) % ny, fz.astype(np.int64) % nz
    xs, ys, zs = (x0, (x0 + 1) % nx), (y0, (y0 + 1) % ny), (z0, (z0 + 1) % nz)
    wx, wy, wz = (1 - ax, ax), (1 - ay, ay), (1 - az, az)
    v = interp(u, shape, x, y, z)
    J = [[np.zeros_like(x) for _ in range(3)] for _ in range(3)]
    for q in range(8):
        bx, by, bz = q & 1, (q >> 1) & 1, q >> 2
        idx = xs[bx] + nx * (ys[by] + ny * zs[bz])
        sx, sy, sz = (1.0 if bx else -1.0), (1.0 if by else -1.0), (1.0 if bz else -1.0)
        for a in range(3):
            uq = u[a][idx]
            J[a][0] = J[a][0] + sx * wy[by] * wz[bz] * uq
            J[a][1] = J[a][1] + sy * wx[bx] * wz[bz] * uq
            J[a][2] = J[a][2] + sz * wx[bx] * wy[by] * uq
    return v, J


def orientations(ids, seed: int):
    """Isotropic unit vectors (3, n): three Philox normals per tracer (counter
    id, step 2^32 - 1, draws 0 and 1), normalised."""
    a, b = normal_pair(seed, ids, 0xFFFFFFFF, 0, 0)
    c, _ = normal_pair(seed, ids, 0xFFFFFFFF, 0, 1)
    g = np.sqrt(a * a + b * b + c * c)
    return np.stack([a / g, b / g, c / g])


def blocked(solid_flat, shape, x, y, z):
    nz, ny, nx = shape
    ix = np.floor(x + 0.5).astype(np.int64) % nx
    iy = np.floor(y + 0.5).astype(np.int64) % ny
    iz = np.floor(z + 0.5).astype(np.int64) % nz
    return solid_flat[ix + nx * (iy + ny * iz)] != 0


def step(pos, dm, ids, u, solid, step_index: int, substeps: int = 1, order: int = 2, seed: int = 0, stretch=None,
         cgrid=None):
    """One lattice step of all tracers; returns (pos, vel), each (3, n). With
    stretch = (rho_hat (3, n), log_rho (n,)) also the new rho_hat, log_rho and
    the step's row (step_index + 1, lambda, mean_log_rho, var_log_rho,
    n_active, lambda_w, lambda_nw, n_w, n_nw); cgrid: node-indexed order
    parameter for the phase split (c < 0.5 wetting), or None."""
    shape = solid.shape
    nz, ny, nx = shape
    sf = np.ascontiguousarray(solid, np.uint8).reshape(-1)
    x, y, z = (np.array(pos[a], np.float64) for a in range(3))
    n = len(x)
    dt = 1.0 / substeps
    kick = np.where(dm > 0.0, np.sqrt(2.0 * np.maximum(dm, 0.0) * dt), 0.0)
    move = kick > 0.0
    if stretch is not None:
        rh = np.array(stretch[0], np.float64).reshape(3, n)
        lr = np.array(stretch[1], np.float64)
        active = np.ones(n, bool)
        lam, lw, lnw, cw, cnw = (np.zeros(n) for _ in range(5))
    for s in range(substeps):
        if stretch is not None:
            k1, J = interp_grad(u, shape, x, y, z)
        else:
            k1 = interp(u, shape, x, y, z)
        if order == 1:
            nxp, nyp, nzp = x + dt * k1[0], y + dt * k1[1], z + dt * k1[2]
        else:
            k2 = interp(u, shape, _wrap(x + dt * k1[0], nx), _wrap(y + dt * k1[1], ny), _wrap(z + dt * k1[2], nz))
            nxp = x + 0.5 * dt * (k1[0] + k2[0])
            nyp = y + 0.5 * dt * (k1[1] + k2[1])
            nzp = z + 0.5 * dt * (k1[2] + k2[2])
        if move.any():
            g0, g1 = normal_pair(seed, ids, step_index, s, 0)
            nxp = np.where(move, nxp + kick * g0, nxp)
            nyp = np.where(move, nyp + kick * g1, nyp)
            if nz > 1:
                g2, _ = normal_pair(seed, ids, step_index, s, 1)
                nzp = np.where(move, nzp + kick * g2, nzp)
        nxp, nyp = _wrap(nxp, nx), _wrap(nyp, ny)
        nzp = _wrap(nzp, nz) if nz > 1 else z  # 2-D: no motion along z
        ok = ~blocked(sf, shape, nxp, nyp, nzp)
        if stretch is not None:
            active &= ok
            jr = [J[i][0] * rh[0] + J[i][1] * rh[1] + J[i][2] * rh[2] for i in range(3)]
            ls = rh[0] * jr[0] + rh[1] * jr[1] + rh[2] * jr[2]
            lam = np.where(ok, lam + ls, lam)
            if cgrid is not None:
                ix = np.floor(x + 0.5).astype(np.int64) % nx
                iy = np.floor(y + 0.5).astype(np.int64) % ny
                iz = np.floor(z + 0.5).astype(np.int64) % nz
                cv = np.asarray(cgrid)[ix + nx * (iy + ny * iz)]
                w, nw = ok & (cv < 0.5), ok & (cv >= 0.5)
                lw, cw = np.where(w, lw + ls, lw), cw + w
                lnw, cnw = np.where(nw, lnw + ls, lnw), cnw + nw
            r = [rh[i] + dt * jr[i] for i in range(3)]
            g = np.sqrt(r[0] * r[0] + r[1] * r[1] + r[2] * r[2])
            lr = np.where(ok, lr + np.log(g), lr)
            rh = np.where(ok, np.stack([r[0] / g, r[1] / g, r[2] / g]), rh)
        x, y, z = np.where(ok, nxp, x), np.where(ok, nyp, y), np.where(ok, nzp, z)
    vel = interp(u, shape, x, y, z)
    if stretch is None:
        return np.stack([x, y, z]), np.stack(vel)
    nact = float(active.sum())
    S = float(substeps)
    sw, sn = float(cw[active].sum()), float(cnw[active].sum())
    mean = lr.sum() / n
    row = np.array([step_index + 1, lam[active].sum() / (nact * S) if nact else np.nan, mean,
                    (lr * lr).sum() / n - mean * mean, nact,
                    lw[active].sum() / sw if sw else np.nan, lnw[active].sum() / sn if sn else np.nan, sw / S, sn / S])
    return np.stack([x, y, z]), np.stack(vel), rh, lr, row
