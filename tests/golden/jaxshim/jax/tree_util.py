"""``jax.tree_util`` functions."""
from ._core import tree_util as _t

register_pytree_node_class = _t.register_pytree_node_class
register_pytree_node = _t.register_pytree_node
tree_map = _t.tree_map
tree_flatten = _t.tree_flatten
tree_unflatten = lambda spec, leaves: _t.tree_unflatten(spec, leaves)
tree_leaves = _t.tree_leaves
