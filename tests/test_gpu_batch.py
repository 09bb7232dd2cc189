"""Batched multi-mesh assembly (one persistent, graph-captured launch) against
the oracle per member, against the per-mesh launch loop (bitwise), and the
FP32-contraction path within 1e-6."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

from dolfin_b200 import synthetic
from dolfin_b200.batch import BatchAssembler, autotune


def _members(count, seed, n_lo=2, n_hi=12):
    specs = synthetic.batched_square_meshes(count, seed, n_lo=n_lo, n_hi=n_hi)
    return specs, [synthetic.build_batch_member(s) for s in specs]


def test_batch_matches_oracle_and_loop(orc):
    specs, built = _members(24, 11)
    members = [(V, k) for (_, V, k, _, _) in built]
    B = BatchAssembler(members)
    mats = [A.values_tensor().clone() for A in B.assemble()]
    torch.cuda.synchronize()
    for A in B.matrices:
        A.values_tensor().zero_()
    loop = [A.values_tensor().clone() for A in B.assemble_loop()]
    torch.cuda.synchronize()
    for a, b in zip(mats, loop):
        assert torch.equal(a, b)
    for spec, (mesh, V, k, x, kv), vals in zip(specs, built, mats):
        om = orc.unit_square_mesh(spec["n"], spec["n"])
        om.coords = x
        od, N = orc.dofmap(om, spec["degree"])
        rp, cols = V.pattern().csr_host()
        ref = orc.assemble_matrix(orc.form(orc.DIFFUSION, 2, spec["degree"], 1, coeff=orc.COEFF_P1),
                                  om, od, od, rp, cols, w=kv)
        got = vals.cpu().numpy()
        scale = np.repeat(np.maximum.reduceat(np.abs(ref), rp[:-1]), np.diff(rp))
        assert np.max(np.abs(got - ref) / scale) <= 1e-12


def test_batch_replay_is_repeatable_and_fp32_close():
    _, built = _members(16, 12)
    members = [(V, k) for (_, V, k, _, _) in built]
    B = BatchAssembler(members, tile_threads=64, seg_cap_bytes=8192)
    first = [A.values_tensor().clone() for A in B.assemble()]
    second = [A.values_tensor().clone() for A in B.assemble()]
    for a, b in zip(first, second):
        assert torch.equal(a, b)
    f32 = [A.values_tensor().clone() for A in B.assemble("fp32")]
    for a, b in zip(first, f32):
        assert float((a - b).abs().max() / a.abs().max()) <= 1e-6


def test_autotune_returns_a_candidate(tmp_path):
    _, built = _members(8, 13)
    members = [(V, k) for (_, V, k, _, _) in built]
    cands = [(64, 8192, 0), (128, 16384, 0)]
    best, timings = autotune(members, candidates=cands, cache_path=str(tmp_path / "tune.json"))
    assert tuple(best) in cands and len(timings) == 2
    best2, _ = autotune(members, candidates=cands, cache_path=str(tmp_path / "tune.json"))
    assert tuple(best2) == tuple(best)  # cached
