"""The Python consumer mirrors: FockBuilder (reference python/src/consumer_bindings.cpp:41-222)
and GpuFockBuilder (python/src/advanced_bindings.cpp:680-749) driven through
Engine.compute / compute_and_consume, as a reference Python user drives them.

CPU: the host builder's own logic (size checks, Fock matrix, reset).
GPU: both builders give the engine's J and K, accumulate across calls until
reset(), and raise the reference's errors."""
import numpy as np
import pytest

TOL = 1e-10  # the J/K parity tolerance of the GPU tests


def test_fock_builder_host_logic(lai):
    n = 4
    fb = lai.FockBuilder(n)
    with pytest.raises(ValueError):
        fb.set_density(np.zeros((n + 1, n + 1)))
    fb.set_density(np.eye(n))
    fb.J[:] = 2.0
    fb.K[:] = 1.0
    H = np.full((n, n), 0.5)
    assert np.allclose(fb.get_fock_matrix(H), 0.5 + 2.0 - 0.5 * 1.0)
    assert np.allclose(fb.get_fock_matrix(H, exchange_fraction=1.0), 0.5 + 2.0 - 1.0)
    fb.reset()
    assert not fb.get_coulomb_matrix().any() and not fb.get_exchange_matrix().any()


def test_operator_and_screening_mirrors(lai):
    assert lai.Operator.coulomb().is_two_electron()
    assert lai.ScreeningOptions.normal().threshold == 1e-12
    assert lai.ScreeningOptions.tight().threshold == 1e-14
    assert lai.ScreeningOptions.loose().threshold == 1e-10
    none = lai.ScreeningOptions.none()
    assert not none.enabled and none.effective_threshold() == 0.0


def _host_only_engine(lai, nbf, threshold):
    # an Engine object without a device handle: enough for the argument checks,
    # which all run before any device call
    import types
    eng = lai.Engine.__new__(lai.Engine)
    eng._h = None
    eng.basis = types.SimpleNamespace(nbf=nbf)
    eng.threshold = threshold
    eng.device = 0
    return eng


def test_compute_and_consume_argument_checks(lai):
    n = 3
    eng = _host_only_engine(lai, n, 1e-12)
    op = lai.Operator.coulomb()
    fb = lai.FockBuilder(n)
    with pytest.raises(RuntimeError):           # density not set
        eng.compute_and_consume(op, fb)
    fb.set_density(np.eye(n))
    with pytest.raises(ValueError):             # not a two-electron operator
        eng.compute_and_consume(lai.engine.Operator("overlap"), fb)
    with pytest.raises(ValueError):             # nbf mismatch
        other = lai.FockBuilder(n + 1)
        other.set_density(np.eye(n + 1))
        eng.compute_and_consume(op, other)
    # the Schwarz cut is the engine's: another threshold, or screening switched off
    # (threshold 0), is refused rather than silently ignored
    for scr in (lai.ScreeningOptions.tight(), lai.ScreeningOptions.none()):
        with pytest.raises(ValueError):
            eng.compute_and_consume(op, fb, scr)
    eng0 = _host_only_engine(lai, n, 0.0)
    eng0._check_screening(lai.ScreeningOptions.none())      # an unscreened engine accepts none()
    eng._check_screening(lai.ScreeningOptions.normal())      # and the default engine normal()


@pytest.mark.gpu
def test_fock_builders_match_engine(lai):
    w = lai.workloads.make("h2o2_ccpvdz")
    n = w.nbf
    eng = lai.Engine(w.basis)
    J0, K0, _ = eng.jk(w.D)
    op = lai.Operator.coulomb()

    fb = lai.FockBuilder(n)
    fb.set_density(w.D)
    eng.compute_and_consume(op, fb)
    assert np.max(np.abs(fb.get_coulomb_matrix() - J0)) < TOL
    assert np.max(np.abs(fb.get_exchange_matrix() - K0)) < TOL

    gfb = lai.GpuFockBuilder(n)
    assert gfb.nbf() == n
    gfb.set_density(w.D)
    eng.compute(op, gfb)
    gfb.synchronize()
    assert np.max(np.abs(gfb.get_coulomb_matrix() - J0)) < TOL
    assert np.max(np.abs(gfb.get_exchange_matrix() - K0)) < TOL
    eng.compute(op, gfb)  # accumulates, like the reference's device J/K
    assert np.max(np.abs(gfb.get_coulomb_matrix() - 2 * J0)) < 2 * TOL
    H = np.eye(n)
    F = gfb.get_fock_matrix(H)  # exchange_fraction defaults to 1.0, as in the reference binding
    assert np.max(np.abs(F - (H + 2 * J0 - 2 * K0))) < 4 * TOL
    gfb.reset()
    assert not gfb.get_coulomb_matrix().any() and not gfb.get_exchange_matrix().any()

    with pytest.raises(RuntimeError):
        eng.compute(op, lai.GpuFockBuilder(n))  # no density set
    wrong = lai.GpuFockBuilder(n + 1)
    wrong.set_density(np.zeros((n + 1, n + 1)))
    with pytest.raises(ValueError):
        eng.compute(op, wrong)
    with pytest.raises(ValueError):
        gfb.set_density(np.zeros((n + 1, n + 1)))
