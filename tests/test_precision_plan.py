"""Host-side planning of the reduced-precision stores (no GPU)."""
import numpy as np
import pytest

import hlr_b200 as hlr


@pytest.mark.parametrize("fixture", ["c1_small", "c2_small"])
def test_store_bytes_by_precision(request, fixture):
    hm = request.getfixturevalue(fixture)
    b64 = hlr.plan_info(hm, precision="f64")["matrix_bytes"]
    b32 = hlr.plan_info(hm, precision="f32")["matrix_bytes"]
    b16 = hlr.plan_info(hm, precision="f16")["matrix_bytes"]
    bbf = hlr.plan_info(hm, precision="bf16")["matrix_bytes"]
    bmx = hlr.plan_info(hm, precision="mixed")["matrix_bytes"]
    bbfp = hlr.plan_info(hm, precision="bfp")["matrix_bytes"]
    assert b32 * 2 == b64
    assert b16 == bbf and b64 / 4 < b16 < b64 / 4 * 1.2  # 16-bit data + one FP32 scale per chunk
    assert b16 < bmx < b32  # dense FP32, low-rank columns FP32 or FP16
    # BFP stores every column whose bit rate is at most 15 in 16 bits (a
    # superset of the FP16 columns of the mixed store), the rest in 24
    assert b16 < bbfp < bmx


def test_mixed_eps_controls_the_mix(c2_small):
    loose = hlr.plan_info(c2_small, precision="mixed", mixed_eps=1e-4)["matrix_bytes"]
    tight = hlr.plan_info(c2_small, precision="mixed", mixed_eps=1e-8)["matrix_bytes"]
    assert loose < tight
    with pytest.raises(hlr.HLRCError):
        hlr.plan_info(c2_small, precision="mixed", mixed_eps=0.0)


def test_mixed_store_never_holds_fp64_columns(c2_small):
    """A tolerance so tight that some columns would want more than FP32
    still gives an all-FP32 store: reduced-precision plans carry packed
    descriptors only, which FP64 kernels must never see."""
    tight = hlr.plan_info(c2_small, precision="mixed", mixed_eps=1e-14)["matrix_bytes"]
    assert tight == hlr.plan_info(c2_small, precision="f32")["matrix_bytes"]


def test_bfp_tolerance_and_24_bit_floor(c2_small):
    with pytest.raises(hlr.HLRCError):
        hlr.plan_info(c2_small, precision="bfp", mixed_eps=0.0)
    # a tolerance no 16-bit column meets: every column and leaf takes 24 bits
    tight = hlr.plan_info(c2_small, precision="bfp", mixed_eps=1e-14)["matrix_bytes"]
    b32 = hlr.plan_info(c2_small, precision="f32")["matrix_bytes"]
    assert 0.75 * b32 < tight < 0.76 * b32     # 3 bytes per entry plus chunk scales


def test_bfp_column_choice_and_accounting():
    # a rank-1 leaf at eps = 1e-2 has VALR tolerance u = 1e-2 >= 2^-15: U and
    # V are one 16-bit chunk each, counted as 2 rows x 2 bytes plus one FP32
    # chunk scale
    ll = hlr.LeafList(2, 2)
    ll.add_lowrank(0, 0, np.array([[1.0], [2.0]]), np.array([[3.0], [1.0]]))
    info = hlr.plan_info(ll, precision="bfp", mixed_eps=1e-2)
    assert info["matrix_bytes"] == 2 * (2 * 2 + 4)


def test_uniform_is_fp64_only(c3_small):
    with pytest.raises(hlr.HLRCError) as e:
        hlr.plan_info(c3_small, uniform=True, precision="f32")
    assert e.value.status == 1


def test_fp16_conversion_is_round_to_nearest_even():
    # exactly representable values survive; the planner's scale is a power of two
    ll = hlr.LeafList(2, 2)
    ll.add_dense(0, 0, np.array([[1.0, -2.5], [0.125, 1024.0]]))
    info = hlr.plan_info(ll, precision="f16")
    assert info["matrix_bytes"] == 2 * 4 + 4


@pytest.mark.parametrize("prec", ["f16", "bf16", "f32", "mixed", "bfp"])
@pytest.mark.parametrize("n,leaf", [(5000, 48), (8200, 64)])
def test_reduced_plans_form_column_streams(prec, n, leaf):
    # plan_info builds the column-stream tables of the multi-vector and
    # 64-vector kernels on the host (every pass segment of one format must be
    # one contiguous run of columns in the store), so a layout that an upload
    # would reject fails here without a GPU
    from conftest import built
    hm = built(f"exp3d_{n}_{leaf}", lambda: hlr.build(hlr.Problem.exp3d(n, leaf_size=leaf)))
    info = hlr.plan_info(hm, precision=prec, max_nrhs=64)
    assert info["matrix_bytes"] > 0
