"""The vecdex-side C++ caller of the C ABI (tests/integration/gpu_searcher.cpp, the GpuSearcher of
INTEGRATION.md), compiled against the reference's own headers and linked with the reference
library and libvdx_b200.so: it builds, maps a failing call to the reference's exception types,
and on a GPU returns exactly what vecdex::HnswIndex::search_batch returns."""

import subprocess
from pathlib import Path

import numpy as np
import pytest

from conftest import integer_matrix, uniform_matrix

GOLDEN = Path(__file__).resolve().parent / "golden"


@pytest.fixture(scope="module")
def program(orc):
    if not orc.build_integration():
        pytest.skip("the integration program needs the reference's headers to be built")
    return orc.INTEGRATION_BIN


def run(program, index, queries, k, ef, workdir):
    qfile = Path(workdir) / "queries.f32"
    np.ascontiguousarray(queries, np.float32).tofile(qfile)
    return subprocess.run([str(program), str(index), str(qfile), str(len(queries)),
                           str(queries.shape[1]), str(k), str(ef)],
                          capture_output=True, text=True, timeout=600)


def test_integration_program_maps_errors_without_a_device(vdx, program, tmp_path):
    """Without a GPU the upload fails: VDX_ERR_CUDA becomes std::runtime_error in the binding."""
    if vdx.device_count() > 0:
        pytest.skip("a device is present")
    res = run(program, GOLDEN / "kat_m8.vdx", integer_matrix(4, 16, 2), 10, 40, tmp_path)
    assert res.returncode == 2 and res.stderr.startswith("error:"), res.stderr


@pytest.mark.gpu
def test_integration_program_equals_the_reference(gpu, orc, program, tmp_path):
    res = run(program, GOLDEN / "kat_m8.vdx", integer_matrix(200, 16, 2), 10, 40, tmp_path)
    assert res.returncode == 0, res.stdout + res.stderr
    assert "differing 0" in res.stdout
    base, queries = uniform_matrix(3000, 40, 21), uniform_matrix(150, 40, 22)
    ref = orc.RefHnsw(40, 2, 12, 80, 9)
    ref.add(base, threads=0)
    ref.save(tmp_path / "cos.vdx")
    for k, ef in ((1, 1), (10, 64)):
        res = run(program, tmp_path / "cos.vdx", queries, k, ef, tmp_path)
        assert res.returncode == 0, res.stdout + res.stderr
