"""Host dictionaries and `.npz` archives of tensors: `convert(Dict, t)` / `convert(TensorMap, d)`
(src/tensors/tensor.jl:433-462). Runs on host tensors; the device round trip is in
test_gpu_storage.py. Every block in the dictionary must equal the oracle's block (the dense
column-major (d₁, d₂) matrix of the coupled sector), and a round trip must reproduce the data
vector exactly."""
import numpy as np
import pytest

from helpers import O, cfg1_spaces, cfg2_spaces, cfg5_spaces, from_sector, to_hom
import tensorkit_b200 as tk
from tensorkit_b200 import storage


def _cases():
    V1, P1 = cfg1_spaces()
    V2, P2 = cfg2_spaces()
    V5, P5 = cfg5_spaces()
    return [("u1", O.randn(O.Hom([V1, P1], [V1]), 0, False)),
            ("su2", O.randn(O.Hom([V2, P2], [V2]), 1, False)),
            ("u1xsu2_complex", O.randn(O.Hom([V5, P5], [V5]), 2, True))]


def _host(t):
    import torch
    return tk.TensorMap(torch.from_numpy(np.ascontiguousarray(t.data)), to_hom(t.W))


@pytest.mark.parametrize("idx", [0, 1, 2])
def test_dict_blocks_match_oracle_and_round_trip(idx):
    _, ot = _cases()[idx]
    t = _host(ot)
    d = tk.to_dict(t)
    assert d["codomain"] == repr(t.space.codomain) and d["domain"] == repr(t.space.domain)
    assert len(d["data"]) == len(t.blocksectors())
    for c in t.blocksectors():
        assert np.array_equal(d["data"][repr(c)], ot.block(from_sector(c)))
    back = tk.from_dict(d)
    assert back.space == t.space and back.data.dtype == t.data.dtype
    assert np.array_equal(back.to_host(), ot.data)


def test_npz_round_trip(tmp_path):
    _, ot = _cases()[2]
    t = _host(ot)
    p = tmp_path / "t.npz"
    storage.save(p, t)
    back = storage.load(p)
    assert back.space == t.space and back.data.dtype == t.data.dtype
    assert np.array_equal(back.to_host(), ot.data)


def test_missing_block_is_zero_and_wrong_shape_is_an_error():
    _, ot = _cases()[1]
    t = _host(ot)
    d = tk.to_dict(t)
    c = t.blocksectors()[0]
    key = repr(c)
    back = tk.from_dict(dict(d, data={k: v for k, v in d["data"].items() if k != key}))
    assert np.count_nonzero(back.block(c).numpy()) == 0
    for c2 in t.blocksectors()[1:]:
        assert np.array_equal(back.block(c2).numpy(), t.block(c2).numpy())
    with pytest.raises(ValueError):
        tk.from_dict(dict(d, data=dict(d["data"], **{key: d["data"][key][:, :-1]})))
    with pytest.raises(ValueError):
        tk.from_dict(dict(d, data=dict(d["data"], **{"SU2Irrep(99)": d["data"][key]})))
