"""felog_load_rmat (the seeded R-MAT stand-in generated on the device) against
the host generator: the CSR built on the device from its own candidates must
equal the CSR of felog_synth_generate's edge list (holdout 0) loaded with
felog_load_graph - same vertex renumbering, same neighbour order, same
weights (bit for bit when uniform; within FP64 rounding when lognormal)."""
import numpy as np
import pytest

import felog_b200 as fb

pytestmark = pytest.mark.gpu


def _host_csr(seed, v_target, e_target, abcd, lognormal, permute):
    g = fb.synth_graph(seed=seed, v_target=v_target, e_target=e_target, abcd=abcd, lognormal=lognormal, holdout=0.0,
                       permute=permute)
    V = g["v_num"]
    f = fb.Felog(v_num=V)
    f.load_graph(g["edges"], V)
    out = f.csr(), V, len(g["edges"]), g["info"]["max_degree"]
    f.close()
    return out


@pytest.mark.parametrize("case", [
    dict(seed=1, v_target=5000, e_target=40000, abcd=(0.57, 0.19, 0.19, 0.05), lognormal=False, permute=True),
    dict(seed=2, v_target=3000, e_target=30000, abcd=(0.6, 0.15, 0.15, 0.1), lognormal=True, permute=True),
    dict(seed=3, v_target=4096, e_target=20000, abcd=(0.57, 0.19, 0.19, 0.05), lognormal=False, permute=False),
    # nearly every pair: the first candidate batch falls short and is drawn again, larger
    dict(seed=4, v_target=64, e_target=1900, abcd=(0.25, 0.25, 0.25, 0.25), lognormal=False, permute=True),
])
def test_device_rmat_equals_host_generator(case):
    (hrow, hnbr, hw), V, E, maxd = _host_csr(**case)
    f = fb.Felog(v_num=V)
    info = f.load_rmat(case["seed"], case["v_target"], case["e_target"], abcd=case["abcd"],
                       lognormal=case["lognormal"], permute=case["permute"])
    assert info["v_num"] == V and info["n_edges"] == E and info["max_degree"] == maxd
    drow, dnbr, dw = f.csr()
    np.testing.assert_array_equal(drow, hrow)
    np.testing.assert_array_equal(dnbr, hnbr)
    if case["lognormal"]:
        np.testing.assert_allclose(dw, hw, rtol=1e-6)
    else:
        np.testing.assert_array_equal(dw, hw)
    f.close()
