"""AMG hierarchy checkpoint (tf_amg_save / tf_amg_load; no reference
counterpart): a restored hierarchy applies with the same bits as the one
that was saved, carries the same statistics and coarse factor, and a file
that does not fit the component, or is cut short, is refused with the
previous hierarchy kept."""
import os

import pytest
import torch

import thermofem_b200 as tf
from conftest import to_device
from thermofem_b200 import problems as P

pytestmark = pytest.mark.gpu

CASES = [("heat3d20", "f32", "v"), ("convdiff16", "f64", "w"), ("heat3d16", "f32v", "f"), ("heat3d20", "f64", "v")]


def _problem(name):
    side = int(name[-2:])
    return P.heat3d(side, seed=3) if name.startswith("heat") else P.convdiff3d(side, seed=49)


@pytest.mark.parametrize("name,hier,cycle", CASES)
def test_restored_hierarchy_applies_the_same_bits(ctx, tmp_path, name, hier, cycle):
    m = _problem(name)
    n = len(m[0]) - 1
    opts = dict(hierarchy_type=hier, cycle=cycle, jacobi_weight=2 / 3, coarse_rows=64)
    a = to_device(m)
    built = tf.Amg(tf.amg_options(**opts), ctx=ctx)
    built.setup(a)
    b = torch.tensor(P.rhs_uniform(n, 5), device="cuda")
    want = built.apply(b).clone()
    path = str(tmp_path / "hierarchy.tfamg")
    built.save(path)
    assert os.path.getsize(path) > 0
    restored = tf.Amg(tf.amg_options(**opts), ctx=ctx)
    restored.load(path)
    assert torch.equal(restored.apply(b), want)
    assert restored.level_statistics() == built.level_statistics()
    assert restored.stop_reason() == built.stop_reason()
    assert restored.coarse_solver() == built.coarse_solver()
    fa, fb = built.coarse_factor(), restored.coarse_factor()
    assert (fa is None) == (fb is None)
    if fa is not None:
        assert torch.equal(fa[0], fb[0]) and torch.equal(fa[1], fb[1])
    for d in range(built.level_count()):
        la, lb = built.level_matrix(d), restored.level_matrix(d)
        assert torch.equal(la.offsets, lb.offsets) and torch.equal(la.indices, lb.indices)
        assert torch.equal(la.values, lb.values)
    # a solver over the restored hierarchy's operator converges as before
    s = tf.Cg(tf.solver_options(), "amg", tf.amg_options(**opts), ctx=ctx) if name.startswith("heat") else None
    if s is not None:
        s.setup(a)
        x = torch.zeros(n, dtype=torch.float64, device="cuda")
        assert s.apply(b, x)["status"] == "Converged"


def test_mismatched_or_damaged_files_are_refused(ctx, tmp_path):
    m = _problem("heat3d16")
    n = len(m[0]) - 1
    a = to_device(m)
    opts = dict(hierarchy_type="f32", jacobi_weight=2 / 3, coarse_rows=64)
    built = tf.Amg(tf.amg_options(**opts), ctx=ctx)
    built.setup(a)
    path = str(tmp_path / "h.tfamg")
    built.save(path)
    b = torch.tensor(P.rhs_uniform(n, 5), device="cuda")
    want = built.apply(b).clone()
    # another hierarchy type, another Jacobi weight
    for other in (dict(opts, hierarchy_type="f64"), dict(opts, jacobi_weight=0.75)):
        c = tf.Amg(tf.amg_options(**other), ctx=ctx)
        with pytest.raises(tf.InvalidArgument):
            c.load(path)
    # a cut file, a foreign file, a missing file: refused, previous hierarchy kept
    data = open(path, "rb").read()
    cut = str(tmp_path / "cut.tfamg")
    with open(cut, "wb") as f:
        f.write(data[: len(data) // 2])
    foreign = str(tmp_path / "foreign.tfamg")
    with open(foreign, "wb") as f:
        f.write(b"not a hierarchy" * 8)
    keep = tf.Amg(tf.amg_options(**opts), ctx=ctx)
    keep.load(path)
    for bad in (cut, foreign, str(tmp_path / "missing.tfamg")):
        with pytest.raises(tf.InvalidArgument):
            keep.load(bad)
        assert torch.equal(keep.apply(b), want)
    # nothing to save before setup
    with pytest.raises(tf.LogicError):
        tf.Amg(tf.amg_options(**opts), ctx=ctx).save(str(tmp_path / "none.tfamg"))
