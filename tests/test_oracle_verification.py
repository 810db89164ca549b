"""The reference's analytic verification checks (tests/verification and
tests/unit of ramc77/SoftFlow), restated against the CPU oracle.  They pin the
oracle to the reference's own known answers, independently of any run of
the reference."""
import math

import numpy as np
import pytest

import oracle as O


def _channel(nx, ny, coll, tau, fx, steps):
    s = O.OracleSim(O.ChannelSpec(nx=nx, ny=ny, collision=coll, tau=tau, body_fx=fx), "sfo")
    s.initialize()
    s.step(steps)
    return s


def _profile_err(s, nx, ny, tau, fx):
    nu = (tau - 0.5) / 3.0
    H = ny - 2
    num = den = q = 0.0
    ux = s.ux()
    for y in range(1, H + 1):
        u = ux[y, nx // 2]
        yp = (y - 1) + 0.5
        ua = (fx / (2.0 * nu)) * yp * (H - yp)
        num += (u - ua) ** 2
        den += ua ** 2
        q += u
    return math.sqrt(num / den), q / (fx * H ** 3 / (12.0 * nu))


def test_poiseuille_bgk():
    """test_poiseuille.cpp:29-79: 16 x 34, fx 1e-6, tau 0.8, 50k steps, L2 < 1 %."""
    s = _channel(16, 34, O.BGK, 0.8, 1e-6, 50000)
    l2, _ = _profile_err(s, 16, 34, 0.8, 1e-6)
    assert l2 < 0.01


@pytest.mark.parametrize("coll", [O.BGK, O.MRT, O.REGULARIZED])
@pytest.mark.parametrize("tau", [0.8, 1.2])
def test_poiseuille_collision_operators(coll, tau):
    """test_poiseuille_collision_operators.cpp:40-132: L2 < 2 %, Q/Q_an within 2 %."""
    nu = (tau - 0.5) / 3.0
    steps = int(5.0 * 32 * 32 / nu)
    s = _channel(8, 34, coll, tau, 1e-6, steps)
    l2, qr = _profile_err(s, 8, 34, tau, 1e-6)
    assert l2 < 0.02 and abs(qr - 1.0) < 0.02


def test_periodic_translation_invariance():
    """test_poiseuille_collision_operators.cpp:142-170: column spread < 1e-10."""
    for nx in (4, 32):
        s = _channel(nx, 34, O.BGK, 0.8, 1e-6, 20000)
        ux = s.ux()[1:-1]
        spread = (ux.max(axis=1) - ux.min(axis=1)).max()
        assert spread / ux.max() < 1e-10


def test_spread_partition_of_unity():
    """test_ibm_momentum_conservation.cpp:97-203: sum F = sum f ds to 1e-12."""
    for nx, ny, cx, cy, R, Nn, f in [(128, 64, 64.0, 32.0, 12.0, 64, (0.001, -0.0007)),
                                    (256, 128, 128.0, 64.0, 16.0, 128, (0.002, 0.001)),
                                    (64, 64, 2.0, 32.0, 5.0, 48, (0.0015, 0.0005))]:
        s = O.OracleSim(O.ChannelSpec(nx=nx, ny=ny), "sfo")
        s.add_capsule(cx, cy, R, Nn, O.Membrane())
        s.initialize()
        P = s.positions()
        s.set_markers(force=np.tile(np.array(f), (len(P), 1)))
        Fx, Fy = s.spread()
        ds = []
        for k in range(len(P)):
            a, b = P[k] - P[k - 1], P[(k + 1) % len(P)] - P[k]
            for d in (a, b):
                if d[0] > nx / 2:
                    d[0] -= nx
                if d[0] < -nx / 2:
                    d[0] += nx
            ds.append(0.5 * (np.hypot(*a) + np.hypot(*b)))
        tot = sum(ds)
        rel = (abs(Fx.sum() - f[0] * tot) + abs(Fy.sum() - f[1] * tot)) / (abs(f[0] * tot) +
                                                                           abs(f[1] * tot))
        assert rel < 1e-12


@pytest.mark.parametrize("model,law", [
    (O.HOOKEAN, lambda l: 0.04 * (l - 1.0)),
    (O.NEO_HOOKEAN, lambda l: 0.01 * (l - 1.0 / l ** 3)),
    (O.SKALAK, lambda l: 0.01 * l * (l * l - 1.0) * 2.0),
])
def test_membrane_tension_laws(model, law):
    """test_membrane_constitutive.cpp:33-86: uniform stretch of a 128-node
    ring, tension = |F| / (2 sin(pi/N)) matches the 1-D law to 1e-10."""
    N, R = 128, 10.0
    for i in range(17):
        lam = 0.8 + 0.05 * i
        if abs(lam - 1.0) < 1e-9:
            continue
        s = O.OracleSim(O.ChannelSpec(nx=200, ny=200), "sfo")
        s.add_capsule(50.0, 50.0, R, N, O.Membrane(model=model, k_stretch=0.04, G_s=0.01,
                                                   C_skalak=1.0, k_bend=0.0, k_area=0.0,
                                                   k_perimeter=0.0, gamma_visc=0.0,
                                                   eta_membrane=0.0))
        s.initialize()
        P = s.positions()
        s.set_markers(pos=np.array([50.0, 50.0]) + (P - np.array([50.0, 50.0])) * lam)
        s.compute_membrane()
        F = s.forces()
        Tm = np.abs(np.hypot(F[:, 0], F[:, 1]).sum() / N / (2.0 * math.sin(math.pi / N)))
        Tr = abs(law(lam))
        assert abs(Tm - Tr) / Tr < 1e-10


def test_helfrich_rest_shape_force_free():
    """test_capsule_bending.cpp:49-60: the circular rest shape is force-free."""
    s = O.OracleSim(O.ChannelSpec(nx=100, ny=100), "sfo")
    s.add_capsule(30.0, 30.0, 8.0, 60, O.Membrane(model=O.HOOKEAN, k_stretch=0.0, k_bend=0.05,
                                                  use_helfrich=1, k_area=0.0, k_perimeter=0.0,
                                                  gamma_visc=0.0, eta_membrane=0.0))
    s.initialize()
    s.compute_membrane()
    assert np.abs(s.forces()).max() < 1e-12


def test_pure_diffusion_variance():
    """test_pure_diffusion.cpp:28-115: sigma^2 = sigma0^2 + 2 D t within 2 %."""
    nx, ny = 256, 8
    s = O.OracleSim(O.ChannelSpec(nx=nx, ny=ny, tau=0.6, periodic_y=1, scalar_enabled=1,
                                  scalar_D=0.05, scalar_periodic_y=1), "sfo")
    s.initialize()
    x = np.arange(nx)
    C0 = np.exp(-((x - nx / 2.0) ** 2) / (2 * 64.0))
    s.set_concentration(np.tile(C0, (ny, 1)))
    s.step(5000)
    c = s.concentration()[0]
    mass = c.sum()
    mean = (c * x).sum() / mass
    var = (c * (x - mean) ** 2).sum() / mass
    expect = 64.0 + 2 * 0.05 * 5000
    assert abs(var - expect) / expect < 0.02
