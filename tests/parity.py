"""Shared helpers of the parity tests: error metrics against the FP64 oracle."""
import numpy as np

# The accuracy bar of the FP32 GPU path against the FP64 oracle: per species, the
# largest absolute difference relative to the largest magnitude of that field.
RTOL = 1e-4


def species_rel_err(gpu, ref):
    """max_v |gpu - ref| / max_v |ref|, per species (fields [species][x][y][z])."""
    out = []
    for s in range(ref.shape[0]):
        scale = np.max(np.abs(ref[s]))
        d = np.max(np.abs(gpu[s] - ref[s]))
        out.append(d / scale if scale > 0 else d)
    return np.array(out)


def pointwise_ok(gpu, ref, rtol=RTOL):
    """|gpu - ref| <= rtol*|ref| + rtol*1e-3*max|ref_s| at every voxel of every species."""
    for s in range(ref.shape[0]):
        floor = rtol * 1e-3 * np.max(np.abs(ref[s]))
        if not np.all(np.abs(gpu[s] - ref[s]) <= rtol * np.abs(ref[s]) + floor):
            return False
    return True


def assert_close(gpu, ref, rtol=RTOL, what=""):
    err = species_rel_err(gpu, ref)
    assert np.all(err <= rtol), f"{what} per-species rel err {err} > {rtol}"
    assert pointwise_ok(gpu, ref, rtol), f"{what} pointwise error above {rtol}"
    return err
