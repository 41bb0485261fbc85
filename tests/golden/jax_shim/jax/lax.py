"""NumPy restatements of the jax.lax control-flow primitives, run eagerly."""


def optimization_barrier(x):
    return x


def cond(pred, true_fun, false_fun, *operands):
    return true_fun(*operands) if bool(pred) else false_fun(*operands)


def while_loop(cond_fun, body_fun, init_val):
    val = init_val
    while bool(cond_fun(val)):
        val = body_fun(val)
    return val


def fori_loop(lower, upper, body_fun, init_val):
    val = init_val
    for i in range(int(lower), int(upper)):
        val = body_fun(i, val)
    return val


def scan(f, init, xs=None, length=None):
    """lax.scan over the leading axis of xs (a pytree of arrays)."""
    import numpy as np

    from . import tree

    carry, ys = init, []
    n = length if xs is None else np.shape(tree.leaves(xs)[0])[0]
    for i in range(n):
        carry, y = f(carry, None if xs is None else tree.map(lambda x: x[i], xs))
        ys.append(y)
    return carry, (np.stack(ys) if ys and ys[0] is not None else None)


def stop_gradient(x):
    return x
