"""A T3 iteration captured as a CUDA graph gives the same t3 and norms as the
eager step, bit for bit, over several replays with inputs changed in place
between them."""
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("precision", ["fp64", "bf16x3"])
def test_graph_replay_matches_eager(precision):
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from dcc import graph, synthetic, t3_residual
    no, nv = 4, 18
    d = synthetic.make_inputs(no, nv, seed=3)
    d.W_oooo = 0.5 * (d.W_oooo + d.W_oooo.permute(1, 0, 3, 2))
    t3_e = d.t3.clone()
    res_e = t3_residual.T3Residual(no, nv, precision, woooo_pair_symmetric=True)
    res_g = t3_residual.T3Residual(no, nv, precision, woooo_pair_symmetric=True)
    t3_g = d.t3.clone()
    g = graph.T3IterationGraph(res_g, d, t3_g)
    t3_g.copy_(d.t3)  # capture ran the step once: restart from the same amplitudes
    norms_e = torch.empty(2, dtype=torch.float64, device="cuda")
    ws = torch.empty(1 << 16, dtype=torch.float64, device="cuda")
    r3 = torch.empty_like(t3_e)
    for it in range(3):
        res_e.compute(d, t3_e, r3)
        t3_residual.update_t3_(t3_e, r3, d, norms=norms_e, workspace=ws, write_r3=False)
        n_g = g.replay()
        torch.cuda.synchronize()
        assert torch.equal(t3_g, t3_e), it
        assert torch.equal(n_g, norms_e), it
        d.t2.mul_(0.99)  # new inputs in the captured buffers
    assert g.status_ok() and res_e.status_ok()
