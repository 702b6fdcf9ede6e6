"""The learned-split MLP's weights file (fkdtree_b200/mlp_file.py): exact
float32 round trip, bfloat16 rounding, header checks.  CPU, plus one GPU
test that a saved network reloads with identical predictions."""
import numpy as np
import pytest

from fkdtree_b200 import mlp_file as M


def _params(seed=0):
    rng = np.random.default_rng(seed)
    p = rng.standard_normal(M.param_count()).astype(np.float32) * np.float32(0.1)
    p[:3] = [0.0, -0.0, 1e-40]  # zeros and a subnormal
    return p


def test_f32_round_trip_is_exact(tmp_path):
    p = _params()
    f = tmp_path / "w.fkdmlp"
    M.save_params(f, p)
    assert f.stat().st_size == M.HEADER + 4 * p.size
    assert np.array_equal(M.load_params(f).view(np.uint32), p.view(np.uint32))


def test_bf16_storage_rounds_to_nearest_even(tmp_path):
    p = _params(1)
    f = tmp_path / "w16.fkdmlp"
    M.save_params(f, p, storage="bf16")
    assert f.stat().st_size == M.HEADER + 2 * p.size
    q = M.load_params(f)
    # the bf16 value nearest to each float32 (ties to even), by brute force over the two neighbours
    b = p.view(np.uint32)
    lo = (b & 0xFFFF0000).view(np.float32)
    hi = ((b & 0xFFFF0000) + 0x10000).view(np.float32)
    dl, dh = np.abs(p.astype(np.float64) - lo), np.abs(hi.astype(np.float64) - p)
    even_lo = ((b >> 16) & 1) == 0
    want = np.where((dl < dh) | ((dl == dh) & even_lo), lo, hi)
    assert np.array_equal(q.view(np.uint32), want.view(np.uint32))
    assert np.array_equal(M.to_bf16_bits(np.array([np.inf, -np.inf], np.float32)), [0x7F80, 0xFF80])
    assert np.isnan(M.from_bf16_bits(M.to_bf16_bits(np.array([np.nan], np.float32))))[0]


def test_header_checks(tmp_path):
    f = tmp_path / "bad"
    f.write_bytes(b"not a weights file" * 8)
    with pytest.raises(ValueError):
        M.load_params(f)
    g = tmp_path / "w"
    M.save_params(g, _params())
    data = bytearray(g.read_bytes())
    data[8] = 9  # version
    (tmp_path / "v").write_bytes(bytes(data))
    with pytest.raises(ValueError):
        M.load_params(tmp_path / "v")
    (tmp_path / "t").write_bytes(g.read_bytes()[:-4])  # truncated
    with pytest.raises(ValueError):
        M.load_params(tmp_path / "t")
    with pytest.raises(ValueError):
        M.save_params(tmp_path / "x", np.zeros(10, np.float32))


@pytest.mark.gpu
def test_saved_network_predicts_the_same(cuda, tmp_path):
    import fkdtree_b200 as F
    m = F.MLP(seed=3)
    x = np.random.default_rng(0).random((256, F.MLP.IN), dtype=np.float32)
    y = m.forward(x)
    m.save(tmp_path / "m.fkdmlp")
    m2 = F.MLP.load(tmp_path / "m.fkdmlp")
    assert np.array_equal(m2.params.view(np.uint32), m.params.view(np.uint32))
    assert np.array_equal(m2.forward(x).view(np.uint32), y.view(np.uint32))
