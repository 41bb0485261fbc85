"""A NumPy-backed stand-in for the few ``jax`` names the reference's tissue modules touch.

Test infrastructure only: ``tests/golden/make_golden.py`` puts this directory first on
``sys.path`` so that the reference's own step (models/surface_pump.py, surface_pump_v3.py) imports
and runs on its ``xp=np`` branch in a container without jax. Nothing in the package imports it.
Traced-only entry points either pass through (jit), run eagerly (vmap: a loop over the leading
axis; ``.at[...].set`` on the slices it hands out) or raise when called (grad, random).
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


class _AtIndexer:
    """``x.at[index]``: ``set`` returns a copy with index set; mode="drop" leaves an
    out-of-range integer index alone, as jax does."""

    def __init__(self, array, index):
        self.array, self.index = array, index

    def set(self, value, mode=None):
        out = _np.array(self.array, copy=True)
        index = self.index
        if mode == "drop" and _np.ndim(index) == 0:
            i = int(index)
            if not -out.shape[0] <= i < out.shape[0]:
                return out.view(AtArray)
        out[index] = value
        return out.view(AtArray)


class _At:
    def __init__(self, array):
        self.array = array

    def __getitem__(self, index):
        return _AtIndexer(self.array, index)


class AtArray(_np.ndarray):
    """An ndarray with jax's functional ``.at[...]`` updates (vmapped slices carry it)."""

    @property
    def at(self):
        return _At(self)


def vmap(fun, in_axes=0, out_axes=0):
    """A loop over the leading axis of every argument leaf (in_axes 0 only), outputs stacked:
    the same values as jax.vmap, one world at a time."""
    if in_axes != 0 or out_axes != 0:
        raise NotImplementedError("the NumPy vmap maps axis 0 only")

    def mapped(*args):
        leaves = tree.leaves(args)
        n = _np.shape(leaves[0])[0]

        def take(i):
            return tree.map(lambda x: _np.asarray(x[i]).view(AtArray)
                            if _np.ndim(x[i]) else _np.asarray(x[i])[()], args)

        outs = [fun(*take(i)) for i in range(n)]
        return tree.map(lambda *xs: _np.stack([_np.asarray(x) for x in xs]), *outs)

    return mapped


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
