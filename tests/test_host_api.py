"""Host-side logic without a GPU: config normalisation, method tables, the C ABI surface."""
import ctypes
import os
import re

import numpy as np
import pytest

import lbmpy_b200 as L
from lbmpy_b200 import _native as N
from lbmpy_b200 import methods as M
from lbmpy_b200.kernel import build_desc
from oracle import oracle_spec as S

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_symbols():
    text = open(os.path.join(ROOT, "include", "lbm_b200.h")).read()
    return sorted(set(re.findall(r"^int\s+(lbm_\w+)\s*\(", text, re.M)))


def test_library_exports_every_declared_symbol():
    lib = ctypes.CDLL(N.LIB_PATH)
    declared = header_symbols()
    assert declared, "no declarations found"
    assert sorted(N.EXPORTS) == declared
    for name in declared:
        assert hasattr(lib, name), name
    assert lib.lbm_version() == 1


def test_plan_descriptor_layout_matches_header():
    # offsets of the C struct (natural alignment) as laid out in include/lbm_b200.h
    assert N.LbmPlanDesc.rates.offset == 24
    assert N.LbmPlanDesc.force_model.offset == 24 + 27 * 8
    assert ctypes.sizeof(N.LbmPlanDesc) % 8 == 0


def test_batch_descriptor_layout_and_host_checks():
    """LbmDomainDesc / LbmBatchTiling match the header; arguments that need no device are refused
    before any CUDA call."""
    assert N.LbmDomainDesc.strides.offset == 24
    assert N.LbmDomainDesc.rates.offset == 72
    assert N.LbmDomainDesc.ubb_velocity.offset == 72 + 27 * 8
    assert ctypes.sizeof(N.LbmDomainDesc) == 72 + 27 * 8 + 12 * 8
    assert ctypes.sizeof(N.LbmBatchTiling) == 16
    common = N.LbmPlanDesc()
    common.stencil = 19
    doms = (N.LbmDomainDesc * 1)()
    h = ctypes.c_void_p()

    def create(n, tiling):
        t = N.LbmBatchTiling(*tiling)
        return N.lib().lbm_batch_create(ctypes.byref(common), doms, n, None, None, 0, None, 0, ctypes.byref(t),
                                        ctypes.byref(h))
    assert create(0, (32, 8, 1, 0)) == N.LBM_E_INVALID
    assert create(1, (32, 16, 1, 0)) == N.LBM_E_INVALID
    assert create(1, (32, 8, 0, 0)) == N.LBM_E_INVALID
    assert "tiling" in N.last_error()
    common.pattern = N.PATTERN_ESOTWIST
    assert create(1, (32, 8, 1, 0)) == N.LBM_E_UNSUPPORTED
    assert N.lib().lbm_batch_sweep(None, 0, None) == N.LBM_E_INVALID
    assert N.lib().lbm_batch_destroy(None) == N.LBM_OK


def test_trt_magic_number_and_delta_equilibrium():
    cfg = L.LBMConfig(stencil=L.Stencil.D3Q19, method=L.Method.TRT, relaxation_rate=1.8)
    assert cfg.relaxation_rates[1] == pytest.approx(0.25806451612903225)
    assert cfg.delta_equilibrium is True
    assert L.LBMConfig(method=L.Method.CUMULANT, compressible=True, stencil=L.Stencil.D3Q27).delta_equilibrium is False
    with pytest.raises(ValueError):
        L.LBMConfig(method=L.Method.CUMULANT, compressible=False)


def test_default_force_models_and_kernel_type_aliases():
    c = L.LBMConfig(stencil=L.Stencil.D3Q27, method=L.Method.CUMULANT, compressible=True, force=(1e-7, 0, 0))
    assert type(c.force_model).__name__ == "CentralMoment"
    t = L.LBMConfig(stencil=L.Stencil.D3Q19, method=L.Method.TRT, force=(1e-7, 0, 0))
    assert type(t.force_model).__name__ == "Guo"
    a = L.LBMConfig(stencil=L.Stencil.D3Q19, kernel_type="aa_odd")
    assert a.streaming_pattern == "aa" and a.timestep == L.Timestep.ODD


def test_legacy_optimization_dict():
    cfg, opt, conf = L.update_with_default_parameters({"stencil": L.Stencil.D3Q19, "relaxation_rate": 1.5},
                                                      {"double_precision": False, "target": "gpu"})
    assert conf.data_type == "float32"
    assert cfg.relaxation_rates == [1.5]


@pytest.mark.parametrize("name", ["D3Q19", "D3Q27"])
def test_product_and_oracle_derive_the_same_mrt_basis(name):
    groups = M.mrt_orthogonal_groups(name)
    nested = S.mrt_orthogonal_nested_moments(name)
    assert [len(g) for g in groups] == [len(g) for g in nested]
    for g, go in zip(groups, nested):
        for p, po in zip(g, go):
            assert p == {e: c for c, e in S.poly_terms(po)}
    rates = [1.7, 1.5] + [1.0, 1.1, 1.2, 1.3][: len(groups) - 4]
    assert M.rates_for_groups(rates, groups, 3) == [r for _, r in S.relaxation_info(rates, nested, 3)]


def test_d3q19_continuous_equilibrium_differs_from_discrete():
    """lbmpy's default continuous_equilibrium changes the D3Q19 equilibrium (not D3Q27)."""
    _, _, qc = M.population_equilibrium("D3Q19", True)
    _, _, qd = M.population_equilibrium("D3Q19", False)
    assert qc != qd
    _, _, qc27 = M.population_equilibrium("D3Q27", True)
    _, _, qd27 = M.population_equilibrium("D3Q27", False)
    assert qc27 == qd27


def test_generated_tables_are_current():
    from lbmpy_b200.csrc import gen_tables
    path = os.path.join(ROOT, "lbmpy_b200", "csrc", "lbm_tables.h")
    assert open(path).read() == gen_tables.generate()


def test_plan_descriptors_of_the_benchmark_configs():
    # D3Q19 TRT FP64 pull periodic
    k = L.create_lb_function(lbm_config=L.LBMConfig(stencil=L.Stencil.D3Q19, method=L.Method.TRT,
                                                    relaxation_rate=1.8, compressible=True))
    d = build_desc(k.update_rule, (64, 64, 64), (1, 1, 1), {})
    assert (d.stencil, d.method, d.store_dtype, d.pattern) == (19, N.METHOD_TRT, N.DTYPE_F64, N.PATTERN_PULL)
    assert d.rates[0] == 1.8 and d.rates[1] == pytest.approx(0.258064516)
    # D3Q27 cumulant FP32 AA with Galilean correction and CentralMoment force
    cfg = L.LBMConfig(stencil=L.Stencil.D3Q27, method=L.Method.CUMULANT, relaxation_rate=1.95, compressible=True,
                      galilean_correction=True, force=(1e-7, 0, 0), streaming_pattern="aa",
                      timestep=L.Timestep.EVEN)
    k = L.create_lb_function(lbm_config=cfg, config=L.CreateKernelConfig(data_type="float32"))
    d = build_desc(k.update_rule, (256, 128, 128), (1, 0, 0), {})
    assert (d.method, d.store_dtype, d.pattern, d.force_model) == (N.METHOD_CUMULANT, N.DTYPE_F32,
                                                                    N.PATTERN_AA, N.FORCE_CENTRAL_MOMENT)
    assert list(d.rates)[4:10] == [1.95] * 5 + [1.0]
    assert d.galilean_correction == 1 and d.force[0] == 1e-7


def test_unsupported_configurations_fail_loudly():
    with pytest.raises(NotImplementedError):
        L.create_lb_method(L.LBMConfig(stencil=L.Stencil.D2Q9, relaxation_rate=1.0))
    with pytest.raises(NotImplementedError):
        L.create_lb_function(lbm_config=L.LBMConfig(stencil=L.Stencil.D3Q19, relaxation_rate=1.0,
                                                    streaming_pattern="esopull", timestep=L.Timestep.EVEN),
                             lbm_optimisation=L.LBMOptimisation(storage_dtype="float16"),
                             config=L.CreateKernelConfig(data_type="float32"))
    with pytest.raises(NotImplementedError):
        L.create_lb_method(L.LBMConfig(stencil=L.Stencil.D3Q19, method=L.Method.CENTRAL_MOMENT, relaxation_rate=1))
    with pytest.raises(ValueError):
        L.create_lb_function(lbm_config=L.LBMConfig(stencil=L.Stencil.D3Q19, relaxation_rate=1.0),
                             lbm_optimisation=L.LBMOptimisation(storage_dtype="float16"))


def test_plan_create_without_a_device_reports_an_error():
    import torch
    if torch.cuda.is_available():
        pytest.skip("device present")
    k = L.create_lb_function(lbm_config=L.LBMConfig(stencil=L.Stencil.D3Q19, relaxation_rate=1.0))
    with pytest.raises(N.LbmError):
        N.Plan(build_desc(k.update_rule, (8, 8, 8), (1, 1, 1), {}))


def test_status_and_variant_queries_check_their_arguments():
    """lbm_plan_status / lbm_sweep_variant refuse NULL plans and outputs before any CUDA call."""
    v = ctypes.c_uint32(7)
    assert N.lib().lbm_plan_status(None, ctypes.byref(v), 1) == N.LBM_E_INVALID
    assert v.value == 7
    out = ctypes.c_int(-1)
    strides = N.i64_array((1, 10, 100, 1000))
    assert N.lib().lbm_sweep_variant(None, None, None, strides, 0, None, ctypes.byref(out)) == N.LBM_E_INVALID
    assert N.lib().lbm_sweep_variant(None, None, None, strides, 0, None, None) == N.LBM_E_INVALID
    assert "NULL" in N.last_error()
