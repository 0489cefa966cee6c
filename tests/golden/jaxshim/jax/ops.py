"""``jax.ops.segment_sum``: scatter-add applied in index order."""
import numpy as _np

from ._core import canon


def segment_sum(data, segment_ids, num_segments=None, **kw):
    data = _np.asarray(data)
    ids = _np.asarray(segment_ids)
    out = _np.zeros((num_segments,) + data.shape[1:], dtype=data.dtype)
    _np.add.at(out, ids, data)
    return canon(out)
