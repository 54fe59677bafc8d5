"""Shared fixtures: markers, the oracle/library bridges and random fields."""

import math
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200) and the built library")
    config.addinivalue_line("markers", "slow: long-running oracle comparison")


def gpu_available():
    try:
        import ctypes
        lib = ctypes.CDLL("libcudart.so")
        n = ctypes.c_int(0)
        return lib.cudaGetDeviceCount(ctypes.byref(n)) == 0 and n.value > 0
    except OSError:
        try:
            import torch
            return torch.cuda.is_available()
        except Exception:
            return False


def pytest_collection_modifyitems(config, items):
    if gpu_available():
        return
    skip = pytest.mark.skip(reason="no CUDA device")
    for it in items:
        if "gpu" in it.keywords:
            it.add_marker(skip)


def rel(a, b):
    """max |a - b| / max |b| (absolute if b is zero)."""
    a = np.asarray(a)
    b = np.asarray(b)
    d = np.abs(a - b).max() if a.size else 0.0
    s = np.abs(b).max() if b.size else 0.0
    return d / s if s > 0 else d


def oracle_grid(cfg):
    from oracle.grid import Grid
    return Grid(cfg.nr, cfg.nth, cfg.nx, cfg.nrchop, cfg.ntchop, cfg.nxchop, cfg.ell, cfg.zlen)


def oracle_physics(cfg):
    from oracle.boussinesq import Physics
    return Physics(dt=cfg.dt, omega=cfg.omega, bv0=cfg.bv0, kappa=cfg.kappa, kappap=cfg.kappap,
                   adams=cfg.adams, visc_sw=cfg.visc_sw, nu=cfg.nu, nup=cfg.nup, p=cfg.p,
                   rmv_sw=getattr(cfg, "rmv_sw", 0))


def random_fff(g, seed, decay=6.0, pad=0, hermitian=True):
    """Band-limited random FFF field (chopped at `pad`), Hermitian at m = 0."""
    from oracle.grid import FFF
    rng = np.random.default_rng(seed)
    A = g.alloc(FFF)
    n = np.arange(g.NRCHOPDIM)[:, None, None]
    A.E = (rng.standard_normal(A.E.shape) + 1j * rng.standard_normal(A.E.shape)) * np.exp(-n / decay)
    if hermitian:
        neg = np.r_[0, np.arange(g.NXCHOPDIM - 1, 0, -1)]
        A.E[:, 0, :] = 0.5 * (A.E[:, 0, :] + np.conj(A.E[:, 0, neg]))
    g.chopset(pad)
    g.chopdo(A)
    g.chopset(-pad)
    return A


def small_cfg(nr=32, nth=16, nx=16, adams=True, **kw):
    from mlegs_b200.inputs import small_config
    return small_config("test_%dx%dx%d" % (nr, nth, nx), nr, nth, nx, adams=adams, **kw)


@pytest.fixture(scope="session")
def lib_built():
    from mlegs_b200 import build
    return build.build()


__all__ = ["rel", "oracle_grid", "oracle_physics", "random_fff", "small_cfg", "math"]
