"""Launch plan of the stage kernels (r3d_gpu_plan, the same function a handle uses at create):
z planes per CTA and column-tile rows, on the host without a GPU."""
import pytest

import r3d_b200 as R

B200_SMS = 148  # the plans below are those of a B200
FP64_HYDRO_CTAS = 3  # resident 128-thread FP64 hydro stage CTAs per SM
MAG = ["--lmag", "1", "--beta", "10", "--rm", "1", "--ampb", "0.1", "--bfh", "2", "--bzp", "20"]


def grid(npx, npy, npz, *extra):
    return ["--npx", str(npx), "--npy", str(npy), "--npz", str(npz), *extra]


@pytest.mark.parametrize("flags,want", [
    (grid(504, 504, 512), (62, 8)),                             # short last chunk (8 x 62 + 16)
    (grid(504, 504, 512, "--precision", "fp32bulk"), (63, 8)),    # four FP32 CTAs per SM
    (grid(504, 504, 2048), (64, 8)),                            # > 64 waves: the tail is negligible
    (grid(504, 504, 64), (15, 8)),                              # 4 x 15 + 4 estimated shorter than 4 x 16
    (grid(32, 32, 64), (4, 8)),                                 # one partial wave: waves x planes
    (grid(126, 126, 256, *MAG), (12, 6)),                       # 32x6 MHD tiles, two CTAs per SM
    (grid(252, 252, 256, *MAG), (12, 6)),
    (grid(64, 64, 128, *MAG), (16, 8)),                         # too few tiles for 32x6
], ids=["fp64_504x504x512", "fp32_504x504x512", "fp64_504x504x2048", "fp64_504x504x64", "fp64_32x32x64",
        "mhd_126x126x256", "mhd_252x252x256", "mhd_64x64x128"])
def test_plan_of_the_measured_grids(flags, want, monkeypatch):
    monkeypatch.delenv("R3D_KCHUNK", raising=False)
    assert R.plan(R.parse(flags), num_sms=B200_SMS) == want


def _default_depth(nloc):
    return 64 if nloc >= 512 else (32 if nloc >= 256 else 16)


@pytest.mark.parametrize("npx,npy", [(504, 504), (252, 252), (96, 64), (1000, 200), (33, 17)])
@pytest.mark.parametrize("npz", [16, 40, 100, 256, 300, 512, 777, 1024])
def test_hydro_depth_bounds(npx, npy, npz, monkeypatch):
    """A hydro depth never exceeds the default; a multi-wave launch adds at most one chunk and
    stays within 3/4 of the default; a single-wave launch takes a power-of-two fraction."""
    monkeypatch.delenv("R3D_KCHUNK", raising=False)
    k, rows = R.plan(R.parse(grid(npx, npy, npz)), num_sms=B200_SMS)
    d = _default_depth(npz)
    assert rows == 8 and 1 <= k <= d
    tiles = -(-npx // 32) * -(-npy // 8)
    if tiles * -(-npz // d) >= FP64_HYDRO_CTAS * 148:
        assert k >= (3 * d + 3) // 4
        assert -(-npz // k) <= -(-npz // d) + 1
    else:
        assert d % k == 0 and k >= 4


def test_slab_plan_and_errors(monkeypatch):
    monkeypatch.delenv("R3D_KCHUNK", raising=False)
    p = R.parse(grid(504, 504, 512))
    assert R.plan(p, 512, B200_SMS) == R.plan(p, 0, B200_SMS)
    k, _ = R.plan(p, 171, B200_SMS)                  # one of three z slabs
    assert 1 <= k <= 16
    for bad in (3, 513):
        with pytest.raises(R.R3dError) as e:
            R.plan(p, bad, B200_SMS)
        assert e.value.code == R.R3D_EINVAL


def test_environment_overrides_depth(monkeypatch):
    p = R.parse(grid(504, 504, 512))
    monkeypatch.setenv("R3D_KCHUNK", "40")
    assert R.plan(p, 0, B200_SMS) == (40, 8)
    monkeypatch.setenv("R3D_KCHUNK", "9999")  # clamped to the planes held
    assert R.plan(p, 0, B200_SMS) == (512, 8)
    for bad in ("0", "12x", "", "-3", "abc"):  # ignored
        monkeypatch.setenv("R3D_KCHUNK", bad)
        assert R.plan(p, 0, B200_SMS) == (62, 8)


def test_plan_follows_the_sm_count(monkeypatch):
    """The plan is computed for the device's SM count: a part with fewer SMs fills its waves
    with fewer CTAs, so a 32x32x64 grid that leaves a B200 mostly idle keeps a deeper chunk on a
    part with 8 SMs, and an MHD grid too small for 32x6 tiles on a B200 takes them there."""
    monkeypatch.delenv("R3D_KCHUNK", raising=False)
    assert R.plan(R.parse(grid(32, 32, 64)), num_sms=B200_SMS) == (4, 8)
    assert R.plan(R.parse(grid(32, 32, 64)), num_sms=8)[0] > 4
    assert R.plan(R.parse(grid(64, 64, 128, *MAG)), num_sms=B200_SMS) == (16, 8)
    assert R.plan(R.parse(grid(64, 64, 128, *MAG)), num_sms=16) == (12, 6)
