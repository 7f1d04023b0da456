"""The oracle's Anderson driver state (checkpoint / resume, one step with a
given G(x)) on the CPU: the restatement of solver_function
(AndersonMixing.jl:56-169) gives the same iterates whether it runs in one call
or is stopped, saved and continued."""
import numpy as np

from oracle.oracle import OracleSystem
from softdft_b200.host.descriptor import numerics_from_dict
from tests.helpers import descriptor, rel, small_slit


def test_resume_equals_uninterrupted():
    ds = small_slit()
    num = numerics_from_dict(dict(ds["numerical"], max_iters=40))
    dft = descriptor(ds)
    whole = OracleSystem(dft.descriptor)
    it, _, _, _ = whole.solve(num)
    assert it == 40
    a = OracleSystem(dft.descriptor)
    a.solve(numerics_from_dict(dict(ds["numerical"], max_iters=15)))
    st, hx, hg = a.solver_state()
    assert st.iter == 15 and st.anderm == num.anderm
    b = OracleSystem(dft.descriptor)
    b.set_x(a.get_x())
    b.set_solver_state(st, hx, hg)
    a.solve_resume(num)
    it_b, _, _ = b.solve_resume(num)
    assert it_b == 40
    assert rel(a.get_x(), whole.get_x()) == 0.0
    assert rel(b.get_x(), whole.get_x()) == 0.0


def test_anderson_step_with_given_objective():
    ds = small_slit()
    dft = descriptor(ds)
    a = OracleSystem(dft.descriptor)
    a.solve(numerics_from_dict(dict(ds["numerical"], max_iters=12)))
    g = a.objective()
    err = a.anderson_step(numerics_from_dict(dict(ds["numerical"], max_iters=100)), g)
    b = OracleSystem(dft.descriptor)
    it, err_b, _, _ = b.solve(numerics_from_dict(dict(ds["numerical"], max_iters=13)))
    assert it == 13 and err == err_b
    assert rel(a.get_x(), b.get_x()) == 0.0
    st, _, _ = a.solver_state()
    assert st.iter == 13 and st.use_picard == 0 and np.any(np.array(st.lambdas[:4]) != 0.0)
