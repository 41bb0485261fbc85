"""A NumPy-backed stand-in for the few ``jax`` names the reference's tissue modules touch.

Test infrastructure only: ``tests/golden/make_golden.py`` puts this directory first on
``sys.path`` so that the reference's own step (models/surface_pump.py, surface_pump_v3.py) imports
and runs on its ``xp=np`` branch in a container without jax. Nothing in the package imports it.
Traced-only entry points (jit, vmap, grad, random) either pass through or raise when called.
"""

import sys as _sys

import numpy as _np

# jax.numpy IS numpy here, so the reference's ``xp is np`` branches (ordered scatters, host
# triangular solves) are the ones that run.
_sys.modules[__name__ + ".numpy"] = _np
numpy = _np

from . import lax, scipy, tree, tree_util  # noqa: E402,F401

Array = _np.ndarray
ShapeDtypeStruct = tuple


class _Config:
    jax_enable_x64 = True
    jax_threefry_partitionable = True

    def update(self, *args, **kwargs):
        return None


config = _Config()


def jit(fun=None, **kwargs):
    if fun is None:
        return lambda f: f
    return fun


def _unavailable(name):
    def call(*args, **kwargs):
        raise NotImplementedError(f"jax.{name} is not available in the NumPy stand-in")

    return call


vmap = _unavailable("vmap")
grad = _unavailable("grad")
jacfwd = _unavailable("jacfwd")
jvp = _unavailable("jvp")
checkpoint = jit


def clear_caches():
    return None


def block_until_ready(x):
    return x


class random:  # noqa: N801 - module-like namespace
    key = staticmethod(_unavailable("random.key"))
    fold_in = staticmethod(_unavailable("random.fold_in"))
    bits = staticmethod(_unavailable("random.bits"))
    key_data = staticmethod(_unavailable("random.key_data"))
    wrap_key_data = staticmethod(_unavailable("random.wrap_key_data"))
