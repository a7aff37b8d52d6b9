"""Rigid-body library kernels and trajectory files: gpt_end_effector_positions against the
reference's own FK file (testfiles/0_0_eepos.traj: end_effector_positions_kernel on every row of
0_0_traj.csv, generateeepos.cu:101-107), gpt_forward_dynamics against the reference's explicit-Euler
trajectories (testfiles/*_traj.csv, dt = 1/64, gravity 0) and the oracle, and gpt_read_csv (the
readCSVToVecVec of runme.cu:18-44) on files written from those rows."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")


# ---------------------------------------------------------------------------
# CPU: the trajectory reader
# ---------------------------------------------------------------------------

def test_read_csv_round_trips_reference_rows(gpt, golden, tmp_path):
    tr = golden["traj_0_1"]
    f = tmp_path / "0_1_traj.csv"
    f.write_text("\n".join(",".join(f"{v:.9g}" for v in row) for row in tr) + "\n")
    got = gpt.read_csv(str(f))
    assert got.shape == tr.shape
    np.testing.assert_array_equal(got, tr.astype(np.float32))


def test_read_csv_edge_cases(gpt, tmp_path):
    f = tmp_path / "a.csv"
    f.write_text("1,2,3,\r\n4,5e-3,-6\n\n")  # trailing comma (no empty field), CRLF, blank line
    np.testing.assert_array_equal(gpt.read_csv(str(f)), np.array([[1, 2, 3], [4, 5e-3, -6]], np.float32))
    g = tmp_path / "ragged.csv"
    g.write_text("1,2,3\n4,5\n")
    with pytest.raises(gpt.GptError):
        gpt.read_csv(str(g))
    with pytest.raises(gpt.GptError):
        gpt.read_csv(str(tmp_path / "missing.csv"))


# ---------------------------------------------------------------------------
# GPU
# ---------------------------------------------------------------------------

def dev(a):
    return torch.as_tensor(np.ascontiguousarray(a, np.float32), device="cuda")


@pytest.mark.gpu
def test_end_effector_positions_match_reference_file(gpt, oracle, golden):
    """All 666 rows of 0_0_traj.csv in one launch (row stride 21): within 3e-5 of the reference's
    printed FK (6 significant digits), the FP32 oracle's bound; a stride-14 state batch gives the
    same values."""
    tr, ee = golden["traj_0_0"], golden["eepos_0_0"]
    got = gpt.end_effector_positions(dev(tr), 21).cpu().numpy()
    assert got.shape == ee.shape
    assert np.abs(got - ee).max() < 3e-5, np.abs(got - ee).max()
    want = np.stack([oracle.fk(r[:7].astype(np.float64)) for r in tr[:50]])
    assert np.abs(got[:50] - want).max() < 3e-5
    got14 = gpt.end_effector_positions(dev(tr[:, :14]), 14).cpu().numpy()
    np.testing.assert_array_equal(got14, got)


@pytest.mark.gpu
def test_forward_dynamics_reproduces_reference_trajectories(gpt, oracle, golden):
    """qd_{k+1} = qd_k + dt FD(x_k, u_k) on the reference's explicit-Euler rollouts (the bound the
    oracle meets, 2e-5), and FD within 1e-5 relative of the FP64 oracle row by row."""
    dt = 1.0 / 64
    for name in ("traj_0_1", "traj_1_2", "traj_2_3", "traj_3_4", "traj_4_0"):
        tr = golden[name]
        qdd = gpt.forward_dynamics(dev(tr), 21).cpu().numpy().astype(np.float64)
        x = tr.astype(np.float64)
        res = np.abs(x[2:, 7:14] - (x[1:-1, 7:14] + dt * qdd[1:-1])).max()
        assert res < 2e-5, (name, res)
        for k in range(0, len(tr), 17):
            want = oracle.fd(x[k, :7], x[k, 7:14], x[k, 14:21])
            assert np.abs(qdd[k] - want).max() <= 1e-5 * max(1.0, np.abs(want).max()), (name, k)


@pytest.mark.gpu
def test_library_kernels_reject_bad_strides(gpt):
    x = torch.zeros(21 * 4, device="cuda")
    with pytest.raises(gpt.GptError):
        gpt.forward_dynamics(x, 14)
    with pytest.raises(gpt.GptError):
        gpt.end_effector_positions(x, 3)


@pytest.mark.gpu
def test_forward_dynamics_gradient_matches_oracle(gpt, oracle, golden):
    """gpt_forward_dynamics_gradient (forwardDynamicsAndGradient) on rows of the reference's
    trajectories against the FP64 oracle's fd_grad: qdd within 1e-5 and each 7 x 7 block of df/du
    within 1e-4 of its largest entry (FP32 tangent inverse dynamics); qdd also agrees with
    gpt_forward_dynamics."""
    tr = np.concatenate([golden["traj_0_1"][::5], golden["traj_3_4"][::5]])
    qdd, df = (t.cpu().numpy().astype(np.float64) for t in gpt.forward_dynamics_gradient(dev(tr), 21))
    qdd_fd = gpt.forward_dynamics(dev(tr), 21).cpu().numpy().astype(np.float64)
    assert np.abs(qdd - qdd_fd).max() <= 1e-5 * max(1.0, np.abs(qdd_fd).max())
    for k, row in enumerate(tr.astype(np.float64)):
        wq, wdf = oracle.fd_grad(row[:7], row[7:14], row[14:21])
        assert np.abs(qdd[k] - wq).max() <= 1e-5 * max(1.0, np.abs(wq).max()), k
        for b in range(3):
            blk = slice(49 * b, 49 * (b + 1))
            assert np.abs(df[k, blk] - wdf[blk]).max() <= 1e-4 * max(1e-3, np.abs(wdf[blk]).max()), (k, b)
