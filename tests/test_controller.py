"""The GPU/CPU solver switch (drape_b200.controller.SimController, the reference's SimController,
libs/session/src/sim_controller.cpp:100-176) and the drape_dump tool with its --backend switch.

Failures are made on the host: a "GPU" backend whose creation, build or N-th frame raises (as the CUDA binding raises
CudaError on DRAPE_DEVICE_ERROR), wrapped around the oracle; the GPU test uses the library's own injected device
failure (drape_cuda_inject_failure), which faults nothing. The CPU backend is the oracle, standing in for the
reference's CpuSolver."""
import os

import numpy as np
import pytest

from drape_b200 import controller as SC
from drape_b200 import drape_dump
from drape_b200 import scenes as S
from drape_b200 import session as SS
from drape_b200.scene import Scene


def patch_scene():
    return Scene([S.centred_sheet(0.04, 0.01, 0.2)], S.sphere_field())


class FlakyGpu:
    """A stand-in GPU Solver: the oracle, raising "cuda: ..." from build or from its `fail_at`-th step."""

    def __init__(self, oracle_mod, fail_build=False, fail_at=None):
        self.inner = oracle_mod.OracleSolver()
        self.fail_build, self.fail_at, self.steps = fail_build, fail_at, 0

    def build(self, scene):
        if self.fail_build:
            raise RuntimeError("cuda: no CUDA device of compute capability 10.0")
        self.inner.build(scene)

    def step(self, *a):
        self.steps += 1
        if self.fail_at is not None and self.steps >= self.fail_at:
            raise RuntimeError("cuda: a grid barrier timed out")
        self.inner.step(*a)

    def __getattr__(self, name):
        return getattr(self.inner, name)


def factory(oracle_mod, **gpu_kw):
    made = []

    def make(backend):
        s = FlakyGpu(oracle_mod, **gpu_kw) if backend == SC.CUDA else oracle_mod.OracleSolver()
        made.append(backend)
        return s
    return make, made


DONE = (SS.STATE_SETTLED, SS.STATE_FAILED, SS.STATE_TIMED_OUT)


def run_to_end(ctl):
    ctl.set_running(True)
    return ctl.wait(lambda s: s.revision > 0 and s.state in DONE and not s.running, timeout=120)


def test_build_failure_on_gpu_falls_back_to_cpu(oracle_mod):
    make, made = factory(oracle_mod, fail_build=True)
    ctl = SC.SimController(SC.SimConfig(scene=patch_scene, garments=("sheet",)), make)
    try:
        st = run_to_end(ctl)
    finally:
        ctl.close()
    assert made == [SC.CUDA, SC.CPU]
    assert st.backend == SC.CPU and not st.gpu_available
    assert st.message.startswith("GPU unavailable: cuda:") and st.message.endswith("; using CPU")
    assert st.state == SS.STATE_SETTLED
    assert ctl.exchange.latest().positions.shape == (25, 3)


def test_step_failure_on_gpu_restarts_the_drape_on_cpu(oracle_mod):
    make, made = factory(oracle_mod, fail_at=5)
    ctl = SC.SimController(SC.SimConfig(scene=patch_scene, garments=("sheet",)), make)
    try:
        st = run_to_end(ctl)
        assert made == [SC.CUDA, SC.CPU]
        assert st.backend == SC.CPU and not st.gpu_available and st.state == SS.STATE_SETTLED
        assert st.message == "GPU failed: cuda: a grid barrier timed out; using CPU"
        assert st.revision == 2  # the drape was rebuilt once, on the CPU
        # The configuration stays on the CPU, and the note stays up on later drapes.
        ctl.reset()
        st = ctl.wait(lambda s: s.revision == 3 and s.state in DONE and not s.running, timeout=120)
        assert made == [SC.CUDA, SC.CPU, SC.CPU]
        assert st.message.startswith("GPU failed:") and st.backend == SC.CPU
    finally:
        ctl.close()


def test_cpu_failure_ends_the_drape_failed(oracle_mod):
    class Broken:
        def __init__(self):
            self.inner = oracle_mod.OracleSolver()

        def step(self, *a):
            raise ValueError("bad step")

        def __getattr__(self, name):
            return getattr(self.inner, name)

    ctl = SC.SimController(SC.SimConfig(scene=patch_scene, garments=("sheet",), backend=SC.CPU), lambda b: Broken())
    try:
        st = run_to_end(ctl)
    finally:
        ctl.close()
    assert st.state == SS.STATE_FAILED and st.message == "bad step" and st.backend == SC.CPU


def test_cuda_factory_without_cpu_solver_refuses_cpu():
    with pytest.raises(ValueError, match="no CPU solver"):
        SC.cuda_factory()(SC.CPU)
    with pytest.raises(ValueError, match="unknown solver backend"):
        SC.cuda_factory()("metal")


def test_drape_dump_cpu_backend_writes_obj(oracle_mod, tmp_path, capsys):
    out = tmp_path / "patch.obj"
    code = drape_dump.main(["--workload", "patch", "--backend", "cpu", "--cpu-solver", "oracle:OracleSolver",
                            "--out", str(out)])
    line = capsys.readouterr().out.strip().splitlines()[-1]
    assert code == 0, line
    assert line.startswith("settled=1 failed=0") and "backend=cpu" in line and "particles=25" in line
    text = out.read_text().splitlines()
    assert sum(t.startswith("v ") for t in text) == 25 and sum(t.startswith("f ") for t in text) == 32


@pytest.mark.gpu
def test_injected_device_failure_falls_back_to_cpu(gpu, oracle_mod):
    """The CUDA solver fails its 4th frame (drape_cuda_inject_failure -> DRAPE_DEVICE_ERROR -> CudaError); the
    controller redoes the drape on the CPU backend and it settles there."""
    def make(backend):
        if backend == SC.CUDA:
            s = gpu.CudaSolver(0)
            s.inject_failure(3)
            return s
        return oracle_mod.OracleSolver()

    ctl = SC.SimController(SC.SimConfig(scene=patch_scene, garments=("sheet",)), make)
    try:
        st = run_to_end(ctl)
    finally:
        ctl.close()
    assert st.backend == SC.CPU and not st.gpu_available and st.state == SS.STATE_SETTLED
    assert st.message.startswith("GPU failed: cuda") and st.revision == 2


@pytest.mark.gpu
def test_drape_dump_cuda_backend(gpu, tmp_path, capsys):
    out = tmp_path / "patch.obj"
    code = drape_dump.main(["--workload", "patch", "--backend", "cuda", "--out", str(out)])
    line = capsys.readouterr().out.strip().splitlines()[-1]
    assert code == 0, line
    assert "backend=cuda" in line and "note" not in line
    assert os.path.getsize(out) > 0
