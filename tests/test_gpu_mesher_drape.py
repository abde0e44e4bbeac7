"""A mesh from the pattern mesher drives the CUDA solver: two sewn square pieces meshed at 1 cm, laid flat above the
test sphere with their seam open, one Assembling frame on the device through the C ABI against the oracle (the FP64
restatement of the reference solver) on the same scene, within 1e-5 m (the reference's Metal-vs-emulator bar)."""
import numpy as np
import pytest

from drape_b200 import mesher as M
from drape_b200 import scenes as S
from drape_b200.scene import Scene, jersey_fabric


def _scene():
    a, b = M.rectangle_piece("front", 0.2, 0.2), M.rectangle_piece("back", 0.2, 0.2)
    pat = M.Pattern([a, b], [M.SeamSpec("side", M.segment_edge(a, "right", "right", False),
                                        M.segment_edge(b, "left", "left", True))])
    mesh = M.build_sim_mesh(pat, 0.01)
    g = M.to_garment(mesh, "pair", [jersey_fabric(), jersey_fabric()], height=0.2,
                     offsets=[(-0.22, -0.1, 0.0), (0.02, -0.1, 0.0)])
    return Scene([g], S.sphere_field()), mesh


@pytest.mark.gpu
def test_meshed_garment_one_frame_matches_oracle(gpu, oracle_mod):
    scene, mesh = _scene()
    s = gpu.CudaSolver(0)
    s.build(scene)
    s.set_phase("pair", 0)
    o = oracle_mod.OracleSolver()
    o.build(scene)
    o.set_phase("pair", 0)
    s.step(1 / 60, 1, 2)
    o.step(1 / 60, 1, 2)
    x = s.positions().astype(np.float64)
    assert x.shape == (len(mesh.rest), 3)
    dev = float(np.abs(x - o.positions()).max())
    assert dev < 1e-5, dev
    # The seam closes: after a few more frames the gap between paired vertices shrinks.
    a, b = mesh.seam_pairs[:, 0], mesh.seam_pairs[:, 1]
    gap0 = float(np.linalg.norm(x[a] - x[b], axis=1).max())
    for _ in range(10):
        s.step(1 / 60, 1, 2)
    x = s.positions().astype(np.float64)
    assert float(np.linalg.norm(x[a] - x[b], axis=1).max()) < gap0
