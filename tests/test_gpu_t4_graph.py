"""One T4 update (compute_r4_tri, projector, divide, norms, t4 += r4) replayed as a CUDA
graph against the same step run eagerly, at the N2 6-31G shape (nocc=7, nvir=11, 161
stored blocks).  The scatters of the OO batch add with atomics, so the two runs agree to
rounding: 1e-12 of the largest |t4| change."""
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("precision", ["fp64", "bf16x3"])
def test_t4_iteration_graph_matches_eager(precision):
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from dcc import graph, synthetic
    d = synthetic.make_t4_inputs(7, 11, seed=3)
    t4_0 = d.t4.clone()
    eager = graph.T4Iteration(d, precision)
    norms_e = eager.step().clone()
    t4_e = d.t4.clone()
    d.t4.copy_(t4_0)
    g = graph.T4IterationGraph(graph.T4Iteration(d, precision))
    assert torch.equal(d.t4, t4_0)  # capture itself leaves t4 as it was
    norms_g = g.replay().clone()
    torch.cuda.synchronize()
    scale = (t4_e - t4_0).abs().max()
    assert scale > 0
    assert (d.t4 - t4_e).abs().max() <= 1e-12 * scale
    assert torch.allclose(norms_g, norms_e, rtol=1e-12, atol=0)
    # a second replay continues from the updated amplitudes, as the next iteration would
    eager2 = graph.T4Iteration(synthetic.make_t4_inputs(7, 11, seed=3), precision)
    eager2.d.t4.copy_(t4_e)
    eager2.step()
    g.replay()
    torch.cuda.synchronize()
    assert (d.t4 - eager2.d.t4).abs().max() <= 1e-12 * scale
