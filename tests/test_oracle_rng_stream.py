"""The oracle's sequential random source, the semantics check of the reference's own:
one mt19937 seeded with rng_seed (simulation.hpp:1173) read through
boost::random::uniform_01<> (a 32-bit output x becomes x / 2^32), drawn in the
reference's order.  The Philox counter policy that the CUDA path shares stays the
default; this mode shows that the oracle consumes the reference's stream draw for draw
where the reference does: n x 6 noise uniforms per RK attempt, cell-major
(mechanics.hpp:2493-2509), and per try of divideCells four angles per mother, then
each mother's length fraction, then the mothers' and the daughters' growth rates, two
uniforms (Box-Muller, utils.hpp:648-655) each (growth.hpp:252-350)."""
import numpy as np

import abm_b200
import oracle_ref as orc


def test_stream_is_mt19937_read_through_uniform_01():
    # the value the C++ standard requires of the 10000th output of a default-seeded mt19937
    u = orc.rng_stream_uniforms(5489, 10000)
    assert u[-1] * 2.0 ** 32 == 4123659995
    # numpy's MT19937 with the same integer seeding, raw 32-bit outputs over 2^32
    raw = np.random.RandomState(42).randint(0, 2 ** 32, size=2000, dtype=np.uint32)
    assert np.array_equal(orc.rng_stream_uniforms(42, 2000), raw / 2.0 ** 32)


def lone_cells(k, spacing=40.0, length=3.0):
    """k horizontal cells along x, `spacing` apart: no pairs, no contact with each other."""
    cells = np.zeros((k, 22))
    cells[:, 0] = np.arange(k)
    cells[:, 1] = spacing * np.arange(k)
    cells[:, 3] = 5.0
    cells[:, 4] = 1.0
    cells[:, 13] = length
    cells[:, 14] = length / 2
    cells[:, 17] = 100.0
    cells[:, 18] = 720.0
    cells[:, 19] = 100.0
    cells[:, 20] = 1
    return cells


def test_noise_is_drawn_cell_major_in_component_order():
    k, seed, dt, amp = 3, 11, 1e-3, 0.5
    cells = lone_cells(k)
    _, p = abm_b200.make_params(no_surface=1, adhesion_mode=0, max_rz_noise=amp)
    o = orc.Oracle(p)
    o.set_cells(cells)
    o.set_rng_stream(seed)
    o.build_neighbors()
    new, _, _ = o.rk_attempt(dt)
    assert o.rng_stream_draws() == 6 * k
    # only the rz noise is on: a free cell moves by dt * noise_z / (eta0 l), and cell i's
    # z noise is the third of its six uniforms
    u = orc.rng_stream_uniforms(seed, 6 * k)
    expect = dt * (-amp + 2 * amp * u[6 * np.arange(k) + 2]) / (cells[:, 17] * cells[:, 13])
    # the displacement is a difference from z = 5: a few ulps of z bound its rounding
    np.testing.assert_allclose(new[:, 3] - cells[:, 3], expect, rtol=1e-9, atol=8 * np.spacing(5.0))
    assert np.array_equal(new[:, 1:3], cells[:, 1:3])


def normal(u, v):
    return np.sqrt(-2 * np.log(u)) * np.cos(2 * np.pi * v)


def test_division_draws_follow_the_reference_order():
    k, seed, R = 5, 3, 0.8
    cells = lone_cells(k, length=5.9)                 # every cell is past Ldiv = 5.6
    _, p = abm_b200.make_params(growth_mean=1.5, growth_std=0.1, daughter_length_std=0.05,
                                daughter_angle_xy_bound=0.3, daughter_angle_z_bound=0.1)
    o = orc.Oracle(p)
    o.set_cells(cells)
    o.set_parents(-np.ones(k, dtype=np.int32))
    o.set_rng_stream(seed)
    tries = o.divide(0.25, 0)
    assert tries == 1                                 # lone mothers: the first try satisfies all
    assert o.rng_stream_draws() == 10 * k
    u = orc.rng_stream_uniforms(seed, 10 * k)
    out = o.cells()
    assert out.shape[0] == 2 * k
    # after 4k angle draws: each mother's length fraction M from (u, v), in mother order
    m = np.arange(k)
    frac = np.clip(0.5 + 0.05 * normal(u[4 * k + 2 * m], u[4 * k + 2 * m + 1]), 0, 1)
    np.testing.assert_allclose(out[:k, 13], frac * (5.9 - 2 * R), rtol=1e-12)
    np.testing.assert_allclose(out[k:, 13], (1 - frac) * (5.9 - 2 * R), rtol=1e-12)
    # then the mothers' growth rates, then the daughters'
    np.testing.assert_allclose(out[:k, 16], 1.5 + 0.1 * normal(u[6 * k + 2 * m], u[6 * k + 2 * m + 1]), rtol=1e-12)
    np.testing.assert_allclose(out[k:, 16], 1.5 + 0.1 * normal(u[8 * k + 2 * m], u[8 * k + 2 * m + 1]), rtol=1e-12)


def test_philox_stays_the_default_and_comes_back():
    cells = lone_cells(4, length=5.9)
    _, p = abm_b200.make_params(growth_mean=1.5, growth_std=0.1, daughter_length_std=0.05,
                                daughter_angle_xy_bound=0.3, daughter_angle_z_bound=0.1)
    out = []
    for stream in (False, True):
        o = orc.Oracle(p)
        o.set_cells(cells)
        o.set_parents(-np.ones(4, dtype=np.int32))
        if stream:
            o.set_rng_stream(9)
            o.set_rng_stream(None)
        o.divide(0.25, 0)
        assert o.rng_stream_draws() == 0
        out.append(o.cells())
    assert np.array_equal(out[0], out[1])


def lone_cells_2d(k, spacing=40.0, length=3.0):
    """k 2-D cells along x, `spacing` apart (ABM-2d column order, indices.hpp)."""
    cells = np.zeros((k, 17))
    cells[:, 0] = np.arange(k)
    cells[:, 1] = spacing * np.arange(k)
    cells[:, 3] = 1.0
    cells[:, 9] = length
    cells[:, 10] = length / 2
    cells[:, 13] = 100.0
    cells[:, 14] = 100.0
    cells[:, 15] = 100.0
    cells[:, 16] = 1
    return cells


def test_2d_noise_is_drawn_cell_major_four_per_cell():
    # 2D/include/mechanics.hpp:1760-1771: (rx, ry, nx, ny) per cell, cells in order
    k, seed, amp = 3, 21, 0.5
    cells = lone_cells_2d(k)
    o = orc.Oracle2D(dict(max_noise=amp, adhesion_mode=0))
    o.set_cells(cells)
    o.set_rng_stream(seed)
    o.build_neighbors()
    new, _, _ = o.rk_attempt(1e-3)
    assert o.rng_stream_draws() == 4 * k
    u = orc.rng_stream_uniforms(seed, 4 * k)
    nx, ny = -amp + 2 * amp * u[4 * np.arange(k)], -amp + 2 * amp * u[4 * np.arange(k) + 1]
    # a lone cell's translational mobility is one scalar: x and y move in the noise's ratio
    dx, dy = new[:, 1] - cells[:, 1], new[:, 2] - cells[:, 2]
    # dx is a difference from x (up to 80 um): a few ulps of x bound its rounding
    np.testing.assert_allclose(dx * ny, dy * nx, rtol=1e-9, atol=8 * np.spacing(cells[:, 1].max()) * amp)
    assert np.all(np.sign(dx) == -np.sign(nx)) or np.all(np.sign(dx) == np.sign(nx))


def test_2d_division_draws_one_angle_per_daughter():
    # 2D/include/growth.hpp:252-335: per try two angles per mother (one per daughter), then
    # the length fractions, then the mothers' and the daughters' growth rates
    k, seed, R, L = 4, 5, 0.8, 5.9
    cells = lone_cells_2d(k, length=L)
    o = orc.Oracle2D(dict(growth_mean=1.5, growth_std=0.1, daughter_length_std=0.05,
                          daughter_angle_xy_bound=0.3, Ldiv=5.6))
    o.set_cells(cells)
    o.set_parents(-np.ones(k, dtype=np.int32))
    o.set_rng_stream(seed)
    nd, tries = o.divide(0.25, 0)
    assert tries == 1
    assert o.rng_stream_draws() == 8 * k
    u = orc.rng_stream_uniforms(seed, 8 * k)
    out = o.cells()
    m = np.arange(k)
    frac = np.clip(0.5 + 0.05 * normal(u[2 * k + 2 * m], u[2 * k + 2 * m + 1]), 0, 1)
    np.testing.assert_allclose(out[:k, 9], frac * (L - 2 * R), rtol=1e-12)
    np.testing.assert_allclose(out[k:, 9], (1 - frac) * (L - 2 * R), rtol=1e-12)
    np.testing.assert_allclose(out[:k, 12], 1.5 + 0.1 * normal(u[4 * k + 2 * m], u[4 * k + 2 * m + 1]), rtol=1e-12)
    np.testing.assert_allclose(out[k:, 12], 1.5 + 0.1 * normal(u[6 * k + 2 * m], u[6 * k + 2 * m + 1]), rtol=1e-12)
    # the daughters' orientations turn by the two drawn angles
    ang1 = -0.3 + 0.6 * u[2 * m]
    ang2 = -0.3 + 0.6 * u[2 * m + 1]
    np.testing.assert_allclose(np.arctan2(out[:k, 4], out[:k, 3]), ang1, atol=1e-12)
    np.testing.assert_allclose(np.arctan2(out[k:, 4], out[k:, 3]), ang2, atol=1e-12)


def test_philox_and_the_reference_stream_give_the_same_division_statistics():
    """Parity with the reference's own draws is statistical: dividing the same 3000 lone
    mothers once under the Philox policy and once under the mt19937 stream gives daughters
    whose length fractions, orientations and growth rates are alike in distribution."""
    from scipy import stats
    k, L, R = 3000, 5.9, 0.8
    cells = lone_cells(k, spacing=20.0, length=L)
    _, p = abm_b200.make_params(growth_mean=1.5, growth_std=0.1, daughter_length_std=0.05,
                                daughter_angle_xy_bound=0.3, daughter_angle_z_bound=0.1, rng_seed=17)
    out = {}
    for source in ("philox", "stream"):
        o = orc.Oracle(p)
        o.set_cells(cells)
        o.set_parents(-np.ones(k, dtype=np.int32))
        if source == "stream":
            o.set_rng_stream(17)
        assert o.divide(0.25, 0) == 1
        c = o.cells()
        out[source] = dict(frac=c[:k, 13] / (L - 2 * R), growth=c[:, 16],
                           azimuth=np.arctan2(c[:, 5], c[:, 4]), tilt=np.arcsin(np.clip(c[:, 6], -1, 1)))
    for key in ("frac", "growth", "azimuth", "tilt"):
        a, b = out["philox"][key], out["stream"][key]
        assert not np.array_equal(a, b)                      # different draws ...
        assert stats.ks_2samp(a, b).pvalue > 1e-3, key       # ... from the same distributions
    # and the distributions the reference asks for
    for src in out.values():
        assert abs(src["frac"].mean() - 0.5) < 5 * 0.05 / np.sqrt(k)
        assert abs(src["growth"].std() - 0.1) < 0.01
        assert np.abs(src["azimuth"]).max() <= 0.3 + 1e-12 and np.abs(src["tilt"]).max() <= 0.1 + 1e-12
