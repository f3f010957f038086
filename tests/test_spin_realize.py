"""shape_realize_spin (host spin realization of principal-axis rotators)
against the reference's own realize_spin (oracle/_ref/libshape_ref.so, via
ref_realize_spin_frames), on the CPU: body matrices and total spin vectors
equal to the last bit, over seeded random spin states with spin-rate drift,
libration, spin impulses before and after the initial epoch, dataset angle
and spin offsets, and epochs at t0 and at an impulse epoch."""
import ctypes as C

import numpy as np
import pytest

from oracle.bindings import Reference
from shape_b200 import ctypes_defs as cd
from shape_b200 import engine as eng


@pytest.fixture(scope="module")
def ref():
    return Reference()


def _reference(ref, spin, t, orb, angleoff, omegaoff):
    n = len(t)
    ae, sp = np.zeros((n, 3, 3)), np.zeros((n, 3))
    t = np.ascontiguousarray(t, dtype=np.float64)
    orb = np.ascontiguousarray(orb, dtype=np.float64)
    ao, oo = np.array(angleoff, dtype=np.float64), np.array(omegaoff, dtype=np.float64)
    rc = ref.lib.ref_realize_spin_frames(C.byref(spin), cd.as_dptr(ao), cd.as_dptr(oo), n, cd.as_dptr(t),
                                         cd.as_dptr(orb), cd.as_dptr(ae), cd.as_dptr(sp))
    assert rc == 0
    return ae, sp


def _random_case(rng, with_impulses, unsorted=False):
    t0 = 2458000.0 + rng.uniform(-5, 5)
    period = rng.uniform(0.1, 2.0)                 # days
    omega = (rng.normal(0, 1e-3), rng.normal(0, 1e-3), 2 * np.pi / period)
    omegadot = (0.0, 0.0, rng.normal(0, 1e-6))
    lib = (rng.uniform(0, 0.05), rng.uniform(0, 20), rng.uniform(0, 2 * np.pi)) if rng.random() < 0.5 else (0, 0, 0)
    imps = []
    if with_impulses:
        for _ in range(int(rng.integers(1, 5))):
            imps.append((t0 + rng.uniform(-4, 4), (0.0, 0.0, rng.normal(0, 0.05))))
        imps.sort(key=lambda x: x[0])
        if unsorted:
            imps = imps[::-1]
    spin = eng.spin_state(1, t0, tuple(rng.uniform(0, 2 * np.pi, 3)), omega, omegadot, imps, lib)
    n = 24
    t = np.sort(t0 + rng.uniform(-6, 6, n))
    t[0] = t0                                       # an epoch at t0
    if imps:
        t[1] = imps[0][0]                           # an epoch at an impulse
    orb = rng.normal(0, 1e-2, (n, 3))
    angleoff = tuple(rng.normal(0, 1e-2, 3))
    omegaoff = tuple(rng.normal(0, 1e-4, 3))
    return spin, t, orb, angleoff, omegaoff


@pytest.mark.parametrize("seed", range(12))
def test_realize_spin_bit_exact(ref, seed):
    rng = np.random.default_rng(900 + seed)
    spin, t, orb, ao, oo = _random_case(rng, with_impulses=seed % 3 != 0, unsorted=seed % 4 == 3)
    ae_r, sp_r = _reference(ref, spin, t, orb, ao, oo)
    ae_g, sp_g = eng.realize_spin(spin, t, orb, ao, oo)
    assert np.array_equal(ae_g, ae_r)
    assert np.array_equal(sp_g, sp_r)
    # a proper rotation
    for m in ae_g:
        assert np.allclose(m @ m.T, np.eye(3), atol=1e-12)


def test_realize_spin_no_offsets_is_the_model_rotation(ref):
    """With no drift, impulses or offsets, psi advances at omega_z and the
    total spin is ae^T omega plus the orbital part."""
    spin = eng.spin_state(1, 100.0, (0.3, 1.1, 0.2), (0.0, 0.0, 6.0))
    t = np.array([100.0, 100.25, 99.5])
    ae, sp = eng.realize_spin(spin, t)
    for k, tk in enumerate(t):
        psi = 0.2 + 6.0 * (tk - 100.0)
        assert np.allclose(np.linalg.det(ae[k]), 1.0)
        assert np.allclose(ae[k][2], [np.sin(1.1) * np.sin(0.3), -np.sin(1.1) * np.cos(0.3), np.cos(1.1)])
        assert np.allclose(ae[k][0, 2], np.sin(psi) * np.sin(1.1))
        assert np.allclose(sp[k], ae[k].T @ [0.0, 0.0, 6.0])
    ae_r, sp_r = _reference(ref, spin, t, np.zeros((3, 3)), (0, 0, 0), (0, 0, 0))
    assert np.array_equal(ae, ae_r) and np.array_equal(sp, sp_r)


def test_realize_spin_errors():
    L = eng.load_library()
    spin = eng.spin_state(0, 0.0, (0, 0, 0), (0, 0, 1.0))          # non-principal-axis
    with pytest.raises(eng.EngineError):
        eng.realize_spin(spin, [0.5])
    spin = eng.spin_state(1, 0.0, (0, 0, 0), (0, 0, 1.0))
    spin.n_impulse = cd.MAX_IMPULSES + 1
    with pytest.raises(eng.EngineError):
        eng.realize_spin(spin, [0.5])
    z = np.zeros(3)
    assert L.shape_realize_spin(None, cd.as_dptr(z), cd.as_dptr(z), 0, None, None, None, None) < 0
