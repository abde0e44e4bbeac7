"""The collision-field bake on the GPU (include/drape_bake.h) through the C ABI: bit-exact against the oracle's serial
restatement of bakeCollisionField (the same FP64 arithmetic in the same order, rounded to float), on a sphere, a
union of spheres, the reference's five-component test body and the tube workloads' capsule-union body; the reference's
own field tests on the device field; its 2 s bake bar."""
import numpy as np
import pytest

from drape_b200 import bake as BK
from drape_b200 import meshes as M

pytestmark = pytest.mark.gpu

CASES = {
    "sphere": lambda: [M.icosphere((0, 0, 0), 0.1, 4)],
    "two_spheres": lambda: [M.icosphere((0.08, 0, 0), 0.1, 4), M.icosphere((-0.08, 0, 0), 0.1, 4)],
    "test_body": M.test_body,
    "capsule_union": M.capsule_union_body,
}


@pytest.mark.parametrize("case", sorted(CASES))
def test_bake_is_bit_exact_against_the_oracle(gpu, oracle_mod, case):
    comps = CASES[case]()
    ref = oracle_mod.bake(comps)
    got = BK.bake_field(comps)
    assert np.allclose(got.origin, ref.origin, rtol=0, atol=0) and tuple(got.dims) == tuple(ref.dims)
    assert np.array_equal(got.values, ref.values), int(np.sum(got.values != ref.values))
    assert (got.values < 0).any() and (got.values == np.float32(0.02)).any()


def test_bake_grid_matches(gpu, oracle_mod):
    comps = M.test_body()
    origin, dims = BK.bake_grid(comps)
    ref = oracle_mod.bake(comps)
    assert np.array_equal(origin, ref.origin) and dims == tuple(ref.dims)


def test_device_field_passes_the_reference_field_tests(gpu):
    f = BK.bake_field([M.icosphere((0, 0, 0), 0.1, 4)])
    rng = np.random.default_rng(7)
    d = rng.standard_normal((2000, 3))
    d /= np.linalg.norm(d, axis=1)[:, None]
    r = 0.1 + rng.uniform(-0.015, 0.015, 2000)
    assert np.abs(f.sample(d * r[:, None]) - (r - 0.1)).max() <= 0.001
    assert abs(f.sample(np.zeros((1, 3)))[0] + 0.02) <= 1e-6
    assert abs(f.sample(np.array([[0.15, 0, 0]]))[0] - 0.02) <= 1e-6


def test_open_mesh_is_rejected(gpu):
    m = M.icosphere((0, 0, 0), 0.1, 2)
    m.triangles = m.triangles[:-1]
    with pytest.raises(ValueError, match="not a closed manifold"):
        BK.bake_field([m])


def test_test_body_bakes_under_two_seconds(gpu):
    """test_collision_perf.cpp:11-19: the test body under 2 s, inside the torso negative."""
    BK.bake_field(M.test_body())  # first call pays the module load
    f = BK.bake_field(M.test_body())
    assert BK.last_ms() < 2000.0
    assert f.sample(np.array([[0.0, 1.2, 0.0]]))[0] < 0


def test_baked_body_drives_the_solver(gpu):
    """A tube on the baked capsule-union body (instead of the sampled analytic one) steps like the solver expects:
    finite state, no penetration beyond the snap tolerance after a few frames."""
    from drape_b200 import scenes as S
    body = BK.bake_field(M.capsule_union_body(), BK.options(cell_size=0.006))
    scene = S.seamed_tube(24, 30, field=body)
    s = gpu.CudaSolver(0)
    s.build(scene)
    for _ in range(20):
        s.step(1 / 60, 1, 2)
    st = s.stats()
    assert not st.has_non_finite and st.max_body_penetration <= 0.002
