from ._core import flatten as _flatten, tree_map, unflatten as _unflatten

map = tree_map  # noqa: A001


def leaves(tree, is_leaf=None):
    return _flatten(tree)[0]


def flatten(tree, is_leaf=None):
    return _flatten(tree)


def unflatten(treedef, leaves_):
    return _unflatten(treedef, leaves_)
