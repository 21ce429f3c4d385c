from ._core import flatten, register, tree_map, unflatten


def register_pytree_node(cls, flatten_func, unflatten_func):
    register(cls, flatten_func, unflatten_func)


def register_pytree_node_class(cls):
    register(cls, lambda x: x.tree_flatten(), lambda aux, ch: cls.tree_unflatten(aux, ch))
    return cls


def tree_flatten(tree, is_leaf=None):
    return flatten(tree)


def tree_unflatten(treedef, leaves):
    return unflatten(treedef, leaves)


def tree_leaves(tree, is_leaf=None):
    return flatten(tree)[0]


class Partial:
    def __init__(self, func, *args, **kw):
        self.func, self.args, self.kw = func, args, kw

    def __call__(self, *a, **k):
        return self.func(*self.args, *a, **{**self.kw, **k})
