"""Device tensors to host dictionaries / `.npz` archives and back (src/tensors/tensor.jl:433-462):
the blocks of a device tensor equal the oracle's, and a tensor reloaded onto the GPU reproduces
the stored data exactly and contracts like the original."""
import numpy as np
import pytest

from helpers import O, cfg2_spaces, from_sector, to_device
import tensorkit_b200 as tk
from tensorkit_b200 import storage

pytestmark = pytest.mark.gpu


def test_device_round_trip(tmp_path):
    V, Pp = cfg2_spaces()
    oa = O.randn(O.Hom([V, Pp], [V]), 5, True)
    a = to_device(oa)
    d = tk.to_dict(a)
    for c in a.blocksectors():
        assert np.array_equal(d["data"][repr(c)], oa.block(from_sector(c)))
    p = tmp_path / "a.npz"
    storage.save(p, a)
    b = storage.load(p, device=a.device)
    assert b.device == a.device and b.space == a.space
    assert np.array_equal(b.to_host(), oa.data)
    # the reloaded tensor is an ordinary device tensor
    n0, n1 = tk.norm(a), tk.norm(b)
    assert n0 == n1
