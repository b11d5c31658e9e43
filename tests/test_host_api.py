"""Host-side behaviour of the warp_md drop-in that needs no GPU: the
System/Selection/Trajectory constructors, the selection grammar, device and
enum parsing, frame subsets, and the errors the reference raises."""
import numpy as np
import pytest

import warp_md
from warp_md import plans


def _system(n=6, positions0=None):
    table = {"name": ["CA", "CB", "N", "CA", "C", "O"][:n], "resname": ["ALA"] * n,
             "resid": [1, 1, 1, 2, 2, 3][:n], "element": ["C", "C", "N", "C", "C", "O"][:n]}
    return warp_md.System.from_arrays(table, positions0=positions0)


def test_selection_grammar():
    s = _system()
    assert s.select("all").indices == [0, 1, 2, 3, 4, 5]
    assert s.select("").indices == [0, 1, 2, 3, 4, 5]
    assert s.select("name CA").indices == [0, 3]
    assert s.select("name CA CB").indices == [0, 1, 3]
    assert s.select("resid 1:2").indices == [0, 1, 2, 3, 4]
    assert s.select("resid 2-3").indices == [3, 4, 5]
    assert s.select("resid 1 3").indices == [0, 1, 2, 5]
    assert s.select("name CA and resid 2").indices == [3]
    assert s.select("not element C").indices == [2, 5]
    assert s.select("(name N or name O) and not resid 3").indices == [2]
    for bad in ("bogus", "name", "resid x", "(name CA", "resid 1 :"):
        with pytest.raises(RuntimeError):
            s.select(bad)
    assert s.select_indices([5, 1]).indices == [5, 1]


def test_from_arrays_validation():
    with pytest.raises(RuntimeError):
        warp_md.System.from_arrays({"name": ["A", "B"], "resid": [1]})
    with pytest.raises(RuntimeError):
        warp_md.System.from_arrays({"resid": [1]})
    s = warp_md.System.from_arrays({"name": ["A", "B"]}, positions0=np.zeros((2, 3)))
    assert s.n_atoms() == 2 and s.positions0.dtype == np.float32


def test_trajectory_from_numpy():
    t = warp_md.Trajectory.from_numpy(np.zeros((4, 3), np.float64))
    assert t.coords.shape == (1, 4, 3) and t.coords.dtype == np.float32
    with pytest.raises(RuntimeError):
        warp_md.Trajectory.from_numpy(np.zeros((2, 4, 2), np.float32))
    with pytest.raises(RuntimeError):
        warp_md.Trajectory.from_numpy(np.zeros((2, 4, 3), np.int32))


def test_parsers():
    assert plans.parse_device("auto") == 0
    assert plans.parse_device("cuda") == 0
    assert plans.parse_device("CUDA:3") == 3
    for bad in ("cuda:", "cuda:x", "cuda:1:2", "tpu"):
        with pytest.raises(RuntimeError):
            plans.parse_device(bad)
    with pytest.raises(warp_md.WarpMdError):
        plans.parse_device("cpu")
    with pytest.raises(RuntimeError, match="reference must be"):
        warp_md.RmsdPlan(_system().select("all"), reference="first")
    with pytest.raises(RuntimeError, match="metric must be"):
        warp_md.PairwiseRmsdPlan(_system().select("all"), metric="bogus")
    with pytest.raises(RuntimeError, match="pbc must be"):
        warp_md.PairwiseRmsdPlan(_system().select("all"), pbc="triclinic")


def test_frame_subset_semantics():
    assert plans.frame_subset(5, None) is None
    assert plans.frame_subset(5, [0, 2]).tolist() == [0, 2]
    assert plans.frame_subset(5, [4, 0, 9]).tolist() == [4, 0]
    assert plans.frame_subset(5, [-1, 0, -6]).tolist() == [4, 0]


def test_plan_input_errors_before_device_work():
    s = _system(positions0=None)
    t = warp_md.Trajectory.from_numpy(np.zeros((2, 5, 3), np.float32))
    with pytest.raises(RuntimeError, match="atom count"):
        warp_md.RmsdPlan(s.select("all")).run(t, s)
    t6 = warp_md.Trajectory.from_numpy(np.zeros((2, 6, 3), np.float32))
    with pytest.raises(RuntimeError, match="no topology reference"):
        warp_md.RmsdPlan(s.select("all"), reference="topology").run(t6, s)
    with pytest.raises(warp_md.WarpMdError):
        warp_md.RmsdPlan(s.select("all"), reference="frame0").run(t6, s, device="cpu")
    # metric "dme" with pbc "orthorhombic" needs per-frame box lengths
    with pytest.raises(warp_md.WarpMdError, match="orthorhombic box required"):
        warp_md.PairwiseRmsdPlan(s.select("all"), metric="dme", pbc="orthorhombic").run(t6, s)
    for bad in (np.ones((3, 3), np.float32), np.ones(4, np.float32), np.ones((5, 3), np.float32)):
        tb = warp_md.Trajectory.from_numpy(np.zeros((2, 6, 3), np.float32), box=bad)
        with pytest.raises(RuntimeError, match="box must"):
            warp_md.PairwiseRmsdPlan(s.select("all"), metric="dme", pbc="orthorhombic").run(tb, s)


def test_synth_shapes_and_seeding():
    fr, ref = warp_md.synth.make_trajectory(50, 4, (0.05, 3.0), seed=3)
    fr2, ref2 = warp_md.synth.make_trajectory(50, 4, (0.05, 3.0), seed=3)
    assert fr.shape == (4, 50, 3) and fr.dtype == np.float32
    np.testing.assert_array_equal(fr, fr2)
    steps = np.linalg.norm(np.diff(ref.astype(np.float64), axis=0), axis=1)
    np.testing.assert_allclose(steps, 3.8, rtol=1e-5)
    d = warp_md.synth.make_drift_trajectory(20, 3, 0.1, seed=1)
    assert d.shape == (3, 20, 3)


def test_dme_box_lengths_per_frame():
    """Box lengths handed to wmd_pairwise_dme: (3,) for every frame, or
    (frames, 3) subset like the coordinates; always C-contiguous float32."""
    t = warp_md.Trajectory.from_numpy(np.zeros((4, 6, 3), np.float32), box=np.array([10.0, 11.0, 12.0]))
    b = plans._dme_boxes(t, 4, None)
    assert b.shape == (4, 3) and b.dtype == np.float32 and b.flags["C_CONTIGUOUS"]
    assert (b == np.array([10, 11, 12], np.float32)).all()
    per = np.arange(12, dtype=np.float64).reshape(4, 3) + 5
    t = warp_md.Trajectory.from_numpy(np.zeros((4, 6, 3), np.float32), box=per)
    sub = plans.frame_subset(4, [3, -4])
    b = plans._dme_boxes(t, 2, sub)
    np.testing.assert_array_equal(b, per[[3, 0]].astype(np.float32))
    assert b.flags["C_CONTIGUOUS"]
