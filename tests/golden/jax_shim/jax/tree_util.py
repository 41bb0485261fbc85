"""jax.tree.map over NamedTuples, tuples, lists and dicts of arrays."""


def _is_leaf(x):
    return not isinstance(x, (tuple, list, dict))


def tree_map(f, tree, *rest):  # noqa: A001 - jax's name
    if isinstance(tree, dict):
        return {k: tree_map(f, tree[k], *(r[k] for r in rest)) for k in tree}
    if isinstance(tree, tuple) and hasattr(tree, "_fields"):
        return type(tree)(*(tree_map(f, *parts) for parts in zip(tree, *rest, strict=True)))
    if isinstance(tree, (tuple, list)):
        return type(tree)(tree_map(f, *parts) for parts in zip(tree, *rest, strict=True))
    return f(tree, *rest)


def leaves(tree):
    if isinstance(tree, dict):
        return [x for k in tree for x in leaves(tree[k])]
    if isinstance(tree, (tuple, list)):
        return [x for part in tree for x in leaves(part)]
    return [tree]


def structure(tree):
    return type(tree)
