"""Generates tests/golden/ref_kernels.npz from the reference's own FP32 kernel bodies.

The reference's libs/sim/kernels/{kernels.h, term_math.h} and libs/sim/src/gpu/emulated_device.cpp are compiled from
the reference sources into oracle/_ref/libref_emulated.so (oracle/Makefile, target `ref`); this script runs them on
seeded inputs and stores inputs and outputs, so the tests can pin the oracle and the CUDA path against the reference
on a machine without the reference sources. Sample generators follow libs/sim/tests/test_term_math.cpp:94-228 and
test_kernels.cpp:37-152 (seeds differ: numpy's generator, not std::mt19937).

Run: python tests/golden/make_golden.py   (needs oracle/_ref built: make -C oracle ref)
"""
from __future__ import annotations

import ctypes as C
import math
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.join(ROOT, "drape-2_b200"))

import oracle as O  # noqa: E402
from drape_b200 import scenes as S  # noqa: E402
from drape_b200.scene import Scene, Settings, field_desc, jersey_fabric, stiff_fabric  # noqa: E402

_f = C.c_float


def fp(a):
    return a.ctypes.data_as(C.POINTER(_f))


def rotation(rng):
    axis = rng.uniform(-1, 1, 3)
    axis /= np.linalg.norm(axis)
    ang = 3 * rng.uniform(-1, 1)
    K = np.array([[0, -axis[2], axis[1]], [axis[2], 0, -axis[0]], [-axis[1], axis[0], 0]])
    return np.eye(3) + math.sin(ang) * K + (1 - math.cos(ang)) * K @ K


def stretch_samples(L, count=200, seed=1234):
    rng = np.random.default_rng(seed)
    fabrics = [jersey_fabric(), stiff_fabric(), S.sheet_fabric()]
    out = dict(x=[], dm=[], area=[], fabric=[], energy=[], grad=[], hess=[], min_edge=[])
    for i in range(count):
        a, b, t = rng.uniform(0.002, 0.02), rng.uniform(0.002, 0.02), rng.uniform(0.6, 2.5)
        r = np.array([[0, 0], [a, 0], [b * math.cos(t), b * math.sin(t)]])
        dmat = np.array([[r[1, 0] - r[0, 0], r[2, 0] - r[0, 0]], [r[1, 1] - r[0, 1], r[2, 1] - r[0, 1]]])
        inv = np.linalg.inv(dmat)
        F = np.array([[1 + rng.uniform(-0.2, 0.3), rng.uniform(-0.2, 0.2)],
                      [rng.uniform(-0.2, 0.2), 1 + rng.uniform(-0.2, 0.3)]])
        R = rotation(rng)
        min_edge = min(a, b, np.linalg.norm(r[2] - r[1]))
        x = np.array([R @ np.array([*(F @ r[k]), rng.uniform(-0.1, 0.1) * min_edge]) for k in range(3)])
        x -= x[0]
        fab = fabrics[i % 3]
        dm = np.array([inv[0, 0], inv[1, 0], inv[0, 1], inv[1, 1]], np.float32)
        xf = x.astype(np.float32).reshape(-1)
        e, g, h = _f(), np.zeros(9, np.float32), np.zeros(81, np.float32)
        L.ref_eval_stretch(fp(xf), fp(dm), float(0.5 * abs(np.linalg.det(dmat))), C.byref(fab.to_c()), 100.0,
                           C.byref(e), fp(g), fp(h))
        out["x"].append(xf)
        out["dm"].append(dm)
        out["area"].append(np.float32(0.5 * abs(np.linalg.det(dmat))))
        out["fabric"].append(i % 3)
        out["energy"].append(e.value)
        out["grad"].append(g)
        out["hess"].append(h)
        out["min_edge"].append(min_edge)
    return {f"stretch_{k}": np.asarray(v) for k, v in out.items()}


def hinge_samples(L, count=200, seed=99):
    rng = np.random.default_rng(seed)
    out = dict(x=[], k=[], rest=[], energy=[], grad=[], hess=[], scale=[])
    for _ in range(count):
        e, h1, h2, phi = rng.uniform(0.002, 0.02), rng.uniform(0.002, 0.02), rng.uniform(0.002, 0.02), rng.uniform(-2.5, 2.5)
        x = np.array([[0.3 * e, h1, 0], [0.6 * e, -h2 * math.cos(phi), h2 * math.sin(phi)], [0, 0, 0], [e, 0, 0]])
        x = x @ rotation(rng).T
        x -= x[0]
        K = 1e-5 * (1 + 10 * (rng.uniform(-1, 1) + 1))
        rest = rng.uniform(-0.5, 0.5)
        xf = x.astype(np.float32).reshape(-1)
        en, g, h = _f(), np.zeros(12, np.float32), np.zeros(144, np.float32)
        L.ref_eval_hinge(fp(xf), K, rest, C.byref(en), fp(g), fp(h))
        out["x"].append(xf)
        out["k"].append(np.float32(K))
        out["rest"].append(np.float32(rest))
        out["energy"].append(en.value)
        out["grad"].append(g)
        out["hess"].append(h)
        out["scale"].append(min(e, h1, h2))
    return {f"hinge_{k}": np.asarray(v) for k, v in out.items()}


def seam_samples(L, count=200, seed=7):
    rng = np.random.default_rng(seed)
    out = dict(x=[], target=[], energy=[], grad=[], hess=[])
    for i in range(count):
        d = rng.uniform(-1, 1, 3)
        x = np.array([[0, 0, 0], rng.uniform(0, 0.03) * d / np.linalg.norm(d)])
        target = 0.0 if i % 3 == 0 else rng.uniform(0, 0.03)
        xf = x.astype(np.float32).reshape(-1)
        en, g, h = _f(), np.zeros(6, np.float32), np.zeros(36, np.float32)
        L.ref_eval_seam(fp(xf), target, 1e4, C.byref(en), fp(g), fp(h))
        out["x"].append(xf)
        out["target"].append(np.float32(target))
        out["energy"].append(en.value)
        out["grad"].append(g)
        out["hess"].append(h)
    return {f"seam_{k}": np.asarray(v) for k, v in out.items()}


def friction_samples(L, count=200, seed=42):
    rng = np.random.default_rng(seed)
    eps = 3e-4 / 60.0
    out = dict(dx=[], n=[], mu=[], energy=[], grad=[], hess=[])
    for _ in range(count):
        n = rng.uniform(-1, 1, 3)
        n /= np.linalg.norm(n)
        d = rng.uniform(-1, 1, 3)
        dx = rng.uniform(0, 3) * eps * d / np.linalg.norm(d)
        mu = rng.uniform(0.001, 0.5)
        dxf, nf = dx.astype(np.float32), n.astype(np.float32)
        en, g, h = _f(), np.zeros(3, np.float32), np.zeros(9, np.float32)
        L.ref_eval_friction(fp(dxf), fp(nf), mu, eps, C.byref(en), fp(g), fp(h))
        out["dx"].append(dxf)
        out["n"].append(nf)
        out["mu"].append(np.float32(mu))
        out["energy"].append(en.value)
        out["grad"].append(g)
        out["hess"].append(h)
    return {f"friction_{k}": np.asarray(v) for k, v in out.items()}


def field_samples(L, count=1000, seed=5):
    rng = np.random.default_rng(seed)
    field = S.sphere_field()
    fd, keep = field_desc(field)
    pts, phi, grad = [], [], []
    for _ in range(count):
        d = rng.uniform(-1, 1, 3)
        p = (rng.uniform(0.12, 0.19) * d / np.linalg.norm(d)).astype(np.float32)
        g = np.zeros(3, np.float32)
        phi.append(L.ref_field_sample(C.byref(fd), fp(p)))
        L.ref_field_gradient(C.byref(fd), fp(p), fp(g))
        pts.append(p)
        grad.append(g)
    # collide / land (test_term_math.cpp:229-250)
    rng = np.random.default_rng(11)
    col_in, col_prev, col_out, land_from, land_to, land_out = [], [], [], [], [], []
    for _ in range(300):
        d = rng.uniform(-1, 1, 3)
        d /= np.linalg.norm(d)
        prev = (0.16 * d).astype(np.float32)
        x = (rng.uniform(0.13, 0.153) * d + rng.uniform(0, 0.004) * rng.uniform(-1, 1, 3)).astype(np.float32)
        xo = x.copy()
        L.ref_collide_body(C.byref(fd), 0.0033, 0.3, fp(prev), fp(xo))
        frm, to = (0.2 * d).astype(np.float32), (0.05 * d).astype(np.float32)
        lo = np.zeros(3, np.float32)
        L.ref_land_on_body(C.byref(fd), 0.0033, fp(frm), fp(to), fp(lo))
        col_in.append(x)
        col_prev.append(prev)
        col_out.append(xo)
        land_from.append(frm)
        land_to.append(to)
        land_out.append(lo)
    return dict(field_points=np.asarray(pts), field_phi=np.asarray(phi, np.float32), field_grad=np.asarray(grad),
                collide_x=np.asarray(col_in), collide_prev=np.asarray(col_prev), collide_out=np.asarray(col_out),
                land_from=np.asarray(land_from), land_to=np.asarray(land_to), land_out=np.asarray(land_out))


def spd_samples(L, count=200, seed=3):
    rng = np.random.default_rng(seed)
    A_all, inv_all, ok_all = [], [], []
    for _ in range(count):
        B = rng.uniform(-1, 1, (3, 3))
        A = (B @ B.T + 0.1 * np.eye(3)).astype(np.float32)
        inv = np.zeros(9, np.float32)
        ok = L.ref_invert_spd3(fp(A.reshape(-1).copy()), fp(inv))
        A_all.append(A.reshape(-1))
        inv_all.append(inv)
        ok_all.append(ok)
    return dict(spd_a=np.asarray(A_all), spd_inv=np.asarray(inv_all), spd_ok=np.asarray(ok_all, np.int32))


def rig(n=40, seed=77, pinned=(3, 17, 29)):
    """A random block-CSR SPD system on n particles (the reference's kernel test rig, test_kernels.cpp:37-116)."""
    rng = np.random.default_rng(seed)
    nb = [set([i]) for i in range(n)]
    for i in range(n):
        for _ in range(3):
            j = int(rng.integers(0, n))
            nb[i].add(j)
            nb[j].add(i)
    M = np.zeros((3 * n, 3 * n))
    for i in range(n):
        for j in sorted(nb[i]):
            if j > i:
                Bk = 0.3 * rng.uniform(-1, 1, (3, 3))
                M[3 * i:3 * i + 3, 3 * j:3 * j + 3] = Bk
                M[3 * j:3 * j + 3, 3 * i:3 * i + 3] = Bk.T
    for i in range(n):
        M[3 * i:3 * i + 3, 3 * i:3 * i + 3] = (6.0 + rng.uniform(-1, 1)) * np.eye(3)
    row_start, cols, blocks = [0], [], []
    for i in range(n):
        for j in sorted(nb[i]):
            cols.append(j)
            blocks.append(M[3 * i:3 * i + 3, 3 * j:3 * j + 3])
        row_start.append(len(cols))
    pin = np.zeros(n, np.uint8)
    pin[list(pinned)] = 1
    A = M.copy()
    for i in pinned:
        A[3 * i:3 * i + 3, :] = 0
        A[:, 3 * i:3 * i + 3] = 0
    b = rng.uniform(-1, 1, (n, 3))
    b[list(pinned)] = 0
    return dict(rig_row_start=np.asarray(row_start, np.uint32), rig_col_index=np.asarray(cols, np.uint32),
                rig_blocks=np.asarray(blocks, np.float32), rig_pinned=pin, rig_dense=A, rig_b=b)


def pcg_sample(L, rg):
    n = len(rg["rig_row_start"]) - 1
    grad = (-rg["rig_b"]).astype(np.float32)
    step, resid, its = O.ref_pcg(rg["rig_row_start"], rg["rig_col_index"], rg["rig_blocks"], rg["rig_pinned"],
                                 np.zeros(n, np.uint8), np.zeros((n, 3), np.float32), grad, 50, 1e-2)
    return dict(rig_ref_step=step, rig_ref_resid=resid, rig_ref_iterations=np.int32(its))


def reduce_sample(L):
    rng = np.random.default_rng(1)
    data = rng.uniform(-1.0, 2.0, 100003).astype(np.float32)
    return dict(reduce_data=data, reduce_ref=np.float32(L.ref_reduce(fp(data), len(data))))


def contact_flags():
    """Reference contact candidates (k_contact_setup) for the sheet-on-sphere start, plus points scattered around
    the threshold phi = r + reach of the capsule union."""
    out = {}
    sc = S.sheet_on_sphere()
    r = O.RefEmulated()
    r.build(sc)
    x = sc.initial_positions().astype(np.float32)
    x[:, 1] -= 0.15  # move the sheet down onto the sphere's top so that candidates exist
    near, nrm, off = r.contact_setup(x)
    out.update(contact_sheet_x=x, contact_sheet_near=near, contact_sheet_normal=nrm, contact_sheet_offset=off)
    tube = S.seamed_tube(16, 20, field_n=64, field_cell=0.008)
    r2 = O.RefEmulated()
    r2.build(tube)
    rng = np.random.default_rng(21)
    x = tube.initial_positions().astype(np.float32)
    # pull every particle toward the torso axis by a random amount so many land near the threshold
    scale = rng.uniform(0.6, 1.0, len(x)).astype(np.float32)
    x[:, 0] *= scale
    x[:, 2] *= scale
    near, nrm, off = r2.contact_setup(x)
    out.update(contact_tube_x=x, contact_tube_near=near, contact_tube_normal=nrm, contact_tube_offset=off)
    return out


def trajectories():
    """Positions of the reference's 32-bit GPU algorithm (EmulatedDevice) after one frame on small scenes."""
    out = {}
    f = jersey_fabric()
    f.damping = 0
    cases = {
        "freefall": (Scene([S.flat_garment("sheet", 0.1, 0.1, 0.02, f)]), 1, 10, None),
        "strip": (S.strip_scene(), 3, 1, None),
        "patch": (Scene([S.centred_sheet(0.004, 0.004, 0.2)], S.sphere_field()), 10, 1, None),
        "sheet": (S.sheet_on_sphere(cg_tolerance=1e-2, max_cg=50), 1, 1, None),
        "pair": (Scene([S.sewn_pair()], settings=Settings(gravity=(0, 0, 0))), 3, 10, ("pair", 0)),
    }
    for name, (sc, frames, sub, phase) in cases.items():
        r = O.RefEmulated()
        r.build(sc)
        if phase:
            r.set_phase(*phase)
        for _ in range(frames):
            r.step(1.0 / 60.0, sub, 2)
        out[f"traj_{name}"] = r.positions().astype(np.float32)
        out[f"traj_{name}_frames"] = np.int32(frames)
        out[f"traj_{name}_substeps"] = np.int32(sub)
    return out


def main():
    O.build(ref=True)
    L = O.ref()
    data = {}
    data.update(stretch_samples(L))
    data.update(hinge_samples(L))
    data.update(seam_samples(L))
    data.update(friction_samples(L))
    data.update(field_samples(L))
    data.update(spd_samples(L))
    rg = rig()
    data.update(rg)
    data.update(pcg_sample(L, rg))
    data.update(reduce_sample(L))
    data.update(contact_flags())
    data.update(trajectories())
    path = os.path.join(HERE, "ref_kernels.npz")
    np.savez_compressed(path, **data)
    print(path, os.path.getsize(path), "bytes")


if __name__ == "__main__":
    main()
