"""Geometry and initial-condition helpers over the C-ABI (geometry.cpp).

Masks are numpy uint8 arrays of shape (nz, ny, nx), 1 = solid, so that the
flat index is x + nx*(y + ny*z) as in the C-ABI.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from ._capi import check, lib

_u8 = C.POINTER(C.c_uint8)
_dp = C.POINTER(C.c_double)


def grf(shape, corr_len: float, porosity: float, seed: int, flow_axis: int = 0, open_flow: bool = False):
    """Gaussian random field medium (largest cluster percolating along flow_axis)."""
    nz, ny, nx = shape
    m = np.empty(shape, np.uint8)
    por = C.c_double()
    check(lib.fe_geom_grf(nx, ny, nz, corr_len, porosity, seed, flow_axis, int(open_flow),
                          m.ctypes.data_as(_u8), C.byref(por)))
    return m, por.value


def cylinders(shape, rmin: float, rmax: float, porosity: float, seed: int, gap: float = 1.0, keep_largest=True):
    """2-D random sequential disc pack, extruded along z."""
    nz, ny, nx = shape
    m = np.empty(shape, np.uint8)
    por = C.c_double()
    check(lib.fe_geom_cylinders(nx, ny, nz, rmin, rmax, porosity, gap, seed, int(keep_largest),
                                m.ctypes.data_as(_u8), C.byref(por)))
    return m, por.value


def spheres(shape, radius: float, max_number: int, distance: float, seed: int):
    nz, ny, nx = shape
    m = np.empty(shape, np.uint8)
    check(lib.fe_geom_spheres(nx, ny, nz, radius, max_number, distance, seed, m.ctypes.data_as(_u8)))
    return m


def pad_open(medium: np.ndarray, flow_axis: int, empty_layers: int, buffer_layers: int):
    """Pad a medium for open inlet/outlet along flow_axis (0=x, 1=y, 2=z)."""
    medium = np.ascontiguousarray(medium, np.uint8)
    mz, my, mx = medium.shape
    dims = (C.c_int * 3)()
    check(lib.fe_geom_pad_open(medium.ctypes.data_as(_u8), mx, my, mz, flow_axis, empty_layers, buffer_layers,
                               dims, None))
    out = np.empty((dims[2], dims[1], dims[0]), np.uint8)
    check(lib.fe_geom_pad_open(medium.ctypes.data_as(_u8), mx, my, mz, flow_axis, empty_layers, buffer_layers,
                               dims, out.ctypes.data_as(_u8)))
    return out


def open_lists(solid: np.ndarray, flow_axis: int, buffer_layers: int, split_axis: int = 0):
    """Inlet, outlet, buffer and buffer-reference site lists (reference order)."""
    solid = np.ascontiguousarray(solid, np.uint8)
    nz, ny, nx = solid.shape
    cnt = (C.c_int32 * 3)()
    check(lib.fe_geom_open_lists(solid.ctypes.data_as(_u8), nx, ny, nz, flow_axis, buffer_layers, split_axis,
                                 cnt, None, None, None, None, None))
    ni, no, nb = cnt[0], cnt[1], cnt[2]
    inl, outl = np.empty(ni, np.int32), np.empty(no, np.int32)
    bv, br = np.empty(nb, np.int32), np.empty(nb, np.int32)
    coord = np.empty(ni, np.float64)
    ip = lambda a: a.ctypes.data_as(C.POINTER(C.c_int32))  # noqa: E731
    check(lib.fe_geom_open_lists(solid.ctypes.data_as(_u8), nx, ny, nz, flow_axis, buffer_layers, split_axis,
                                 cnt, ip(inl), ip(outl), ip(bv), ip(br), coord.ctypes.data_as(_dp)))
    return inl, outl, bv, br, coord


def tiff_stack(source, extension: str = "tif", solid_nonzero: bool = True, invert: bool = False,
               coarsening_levels: int = 0, subvolume=None) -> np.ndarray:
    """Solid mask (nz, ny, nx) of a segmented TIFF stack (reference
    domain_geometry = 3d_image). source: a directory (every *.extension file
    in it, in name order, as the reference's image_dir) or a list of files.
    subvolume: (x0, y0, z0, sx, sy, sz) in full-resolution voxels."""
    import os
    if isinstance(source, (str, os.PathLike)) and os.path.isdir(source):
        files = sorted(os.path.join(source, f) for f in os.listdir(source) if f.endswith("." + extension))
    elif isinstance(source, (str, os.PathLike)):
        files = [str(source)]
    else:
        files = [str(f) for f in source]
    if not files:
        raise ValueError(f"no *.{extension} file in {source}")
    arr = (C.c_char_p * len(files))(*[f.encode() for f in files])
    sub = None
    if subvolume is not None:
        sub = (C.c_int32 * 6)(*[int(v) for v in subvolume])
    dims = (C.c_int32 * 3)()
    args = (arr, len(files), int(solid_nonzero), int(invert), int(coarsening_levels), sub, dims)
    check(lib.fe_geom_tiff_stack(*args, None, 0))
    nx, ny, nz = dims
    out = np.empty((nz, ny, nx), np.uint8)
    check(lib.fe_geom_tiff_stack(*args, out.ctypes.data_as(C.POINTER(C.c_uint8)), out.size))
    return out


def site_nodes(solid: np.ndarray) -> np.ndarray:
    solid = np.ascontiguousarray(solid, np.uint8)
    nz, ny, nx = solid.shape
    n = C.c_int64()
    check(lib.fe_geom_sites(solid.ctypes.data_as(_u8), nx, ny, nz, C.byref(n), None))
    nodes = np.empty(n.value, np.int64)
    check(lib.fe_geom_sites(solid.ctypes.data_as(_u8), nx, ny, nz, C.byref(n),
                            nodes.ctypes.data_as(C.POINTER(C.c_int64))))
    return nodes


def order_parameter(solid: np.ndarray, kind: str, width: float, **a) -> np.ndarray:
    """c per site: kind 'uniform' (c), 'slab' (origin, axis, thickness),
    'droplet' (centre, radius); tanh profile (1 + tanh(2 d / width)) / 2."""
    solid = np.ascontiguousarray(solid, np.uint8)
    nz, ny, nx = solid.shape
    if kind == "uniform":
        k, args = 0, [a.get("c", 0.0), 0, 0, 0, 0]
    elif kind == "slab":
        o = a.get("origin", (0.0, 0.0, 0.0))
        k, args = 1, [o[0], o[1], o[2], float(a.get("axis", 0)), float(a["thickness"])]
    elif kind == "droplet":
        cc = a["centre"]
        k, args = 2, [cc[0], cc[1], cc[2], float(a["radius"]), 0.0]
    else:
        raise ValueError(kind)
    n = len(site_nodes(solid))
    out = np.empty(n, np.float64)
    arr = np.array(args, np.float64)
    check(lib.fe_init_order_parameter(solid.ctypes.data_as(_u8), nx, ny, nz, k, arr.ctypes.data_as(_dp), width,
                                      out.ctypes.data_as(_dp)))
    return out


def equilibrium(c: np.ndarray, p, rho0: float, rho1: float, u=None):
    """Plain equilibrium h, g (reference layout f[k*n+i]) of per-site fields."""
    c = np.ascontiguousarray(c, np.float64)
    n = len(c)
    p = np.ascontiguousarray(np.broadcast_to(np.asarray(p, np.float64), (n,)))
    h = np.empty(19 * n, np.float64)
    g = np.empty(19 * n, np.float64)
    if u is None:
        uxp = uyp = uzp = None
    else:
        ux, uy, uz = (np.ascontiguousarray(v, np.float64) for v in u)
        uxp, uyp, uzp = (v.ctypes.data_as(_dp) for v in (ux, uy, uz))
    check(lib.fe_init_equilibrium(n, c.ctypes.data_as(_dp), p.ctypes.data_as(_dp), uxp, uyp, uzp, rho0, rho1,
                                  h.ctypes.data_as(_dp), g.ctypes.data_as(_dp)))
    return h, g
