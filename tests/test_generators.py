"""The seeded generators plant a true optimum: the planted point is feasible
and its KKT score on the reference's own measure is at round-off."""
import numpy as np

from optimisation_solver_b200 import generators as g


def test_reference_lp_shape_and_planted_optimum(oracle):
    p = g.reference_lp(0)
    assert (p.lp.num_rows, p.lp.num_cols, p.lp.nnz) == (1000, 2000, 8000)
    m = oracle.evaluate(p.lp, p.x, -p.y)
    assert m["kkt"] < 1e-12
    assert abs(m["primal_objective"] - p.objective) < 1e-9 * abs(p.objective)


def test_stress_generator_planted_optimum(oracle):
    p = g.planted_lp(400, 800, 6, seed=3, magnitudes="loguniform", free_fraction=0.2,
                     ranged_fraction=0.1, rescale=(-4.0, 4.0))
    m = oracle.evaluate(p.lp, p.x, -p.y)
    assert m["kkt"] < 1e-9
    assert np.isinf(p.lp.var_lower).mean() > 0.1


def test_flow_family_feasible_and_shaped():
    G = g.flow_graph()
    assert G.nodes == 2000 and G.arcs == 20000 and G.incidence.nonzeros == 40000
    s, c = g.flow_parameters(G, 4, 0)
    assert np.allclose(s.sum(axis=1), 0.0, atol=1e-8)
    assert (c > 0).all()


def test_generators_are_seeded():
    a, b = g.reference_lp(5), g.reference_lp(5)
    assert np.array_equal(a.lp.values, b.lp.values) and np.array_equal(a.lp.objective, b.lp.objective)
