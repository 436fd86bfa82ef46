"""Host-side checks of the compiled-form layer (no GPU): the argument checks of FormAssembler2D
(include/femd/forms/assembler_2d.hpp:38-150) and of the solver dispatch raise before any device
work, with the reference's messages."""
import math

import pytest


@pytest.fixture(scope="module")
def fbv():
    import femd_b200 as fb
    m = fb.rectangle_mesh(0, 0, 1, 1, 4, 4)
    V = fb.LagrangeSpace2D(m, 2, bc="dirichlet")
    return fb, V


def test_assembler_argument_checks(fbv):
    fb, V = fbv
    from femd_b200.forms import FormAssembler2D, Integrand
    Q = V.cache(4)
    with pytest.raises(ValueError, match="rank is 1 or 2"):
        FormAssembler2D(3, 0, 0)
    A = FormAssembler2D(2, 1, 2)
    with pytest.raises(ValueError, match="vector index out of range"):
        A.add_field(Q, 1, 0, V.dim, [0])
    with pytest.raises(ValueError, match="dim != the dimension"):
        A.add_field(Q, 0, 0, V.dim + 1, [0])
    with pytest.raises(ValueError, match="no derivative codes"):
        A.add_field(Q, 0, 0, V.dim, [])
    with pytest.raises(ValueError, match="derivative code out of range"):
        A.add_field(Q, 0, 0, V.dim, [3])
    first = A.add_field(Q, 0, 0, V.dim, [0, 1, 2])
    assert first == 0 and A.nval == 3
    with pytest.raises(ValueError, match="needs the trial cache"):
        A.add_group(Q)
    g = A.add_group(Q, Q)
    with pytest.raises(ValueError, match="no such group"):
        A.add_term(5, Integrand.constant(), [], [0], 1, 1)
    with pytest.raises(ValueError, match="takes 1 inputs"):
        A.add_term(g, Integrand.field(), [], [], 1, 1)
    with pytest.raises(ValueError, match="input out of range"):
        A.add_term(g, Integrand.field(), [7], [], 1, 1)
    with pytest.raises(ValueError, match="constant out of range"):
        A.add_term(g, Integrand.constant(), [], [9], 1, 1)
    with pytest.raises(ValueError, match="trial code out of range"):
        A.add_term(g, Integrand.constant(), [], [0], 1, 4)
    with pytest.raises(ValueError, match="reads the normal on a cell group"):
        A.add_term(g, Integrand([[3, 0, 1, 0]], 1, 0, 0), [], [], 0, 0)
    A.add_term(g, Integrand.varcoef(), [], [0, 1, 1], 1, 1)
    assert len(A.groups[g]["terms"]) == 1


def test_integrand_programs(fbv):
    from femd_b200.forms import Integrand
    p = Integrand.varcoef(2 * math.pi)
    assert p.code.shape == (12, 4) and p.nreg == 5 and p.nconst == 3 and p.ninput == 0
    assert p.needs_coordinates and not p.needs_normal
    assert not Integrand.field().needs_coordinates
