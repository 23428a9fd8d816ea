"""Without a CUDA device or without the native library the product path
raises; it never falls back to a CPU solver.  (Runs where no GPU is
visible; on a GPU host these cases cannot be staged and are skipped.)"""
import pytest

from tests.conftest import cuda_available

no_gpu = pytest.mark.skipif(cuda_available(), reason="needs a host without a CUDA device")


@no_gpu
def test_engine_requires_a_cuda_device():
    from co_cultivation_metabolic_atlas_b200 import synthetic as syn
    from co_cultivation_metabolic_atlas_b200.engine import LPEngine
    model, _, _ = syn.single_species_workload(1, m=120, n=260)
    with pytest.raises(RuntimeError, match="no CPU fallback"):
        LPEngine([(model.S, model.S.shape[0])])


@no_gpu
def test_backend_refuses_to_start_without_a_gpu(forbid_cpu_optimizers):
    from co_cultivation_metabolic_atlas_b200 import B200LPBackend
    with pytest.raises(RuntimeError, match="no CPU fallback"):
        B200LPBackend(mode="cold")


def test_missing_native_library_is_an_import_error(tmp_path):
    from co_cultivation_metabolic_atlas_b200 import _native as N
    with pytest.raises(ImportError, match="missing"):
        N.load(tmp_path / "libfbalp.so")
