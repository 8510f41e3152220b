"""Comparison helpers shared by the parity tests."""
import numpy as np

# Halo property tolerance: 1e-6 relative (the bar the GPU path is held to
# against the FP64 oracle).  Mean velocities can sit near zero, so their error
# is normalised by max(|ref|, sigma_v / sqrt(n)), sigma_v = 300 km/s.
PROP_RTOL = 1e-6
SIGMA_V = 300.0


def prop_errors(got, ref):
    """Max normalised error per column of the 7 leading record entries."""
    got = np.asarray(got, np.float64)
    ref = np.asarray(ref, np.float64)
    n = np.maximum(ref[:, 0], 1.0)
    err = np.zeros(7)
    if ref.shape[0] == 0:
        return err
    err[0] = np.max(np.abs(got[:, 0] - ref[:, 0]))
    for c in range(1, 4):
        err[c] = np.max(np.abs(got[:, c] - ref[:, c]) / np.maximum(np.abs(ref[:, c]), 1e-30))
    for c in range(4, 7):
        scale = np.maximum(np.abs(ref[:, c]), SIGMA_V / np.sqrt(n))
        err[c] = np.max(np.abs(got[:, c] - ref[:, c]) / scale)
    return err


def assert_same_catalog(cat, ref, check_member=True):
    """Exact membership and order; properties within PROP_RTOL."""
    nh = ref["halo_head"].shape[0]
    assert cat.nhalos == nh, (cat.nhalos, nh)
    np.testing.assert_array_equal(cat.head, ref["halo_head"])
    np.testing.assert_array_equal(cat.props[:, 0], ref["halo_props"][:, 0])
    err = prop_errors(cat.props[:, :7], ref["halo_props"][:, :7])
    assert err[0] == 0
    assert np.all(err[1:] <= PROP_RTOL), err
    if check_member:
        np.testing.assert_array_equal(cat.member, ref["member"])
