"""The byte counts the roofline figures are quoted on (CPU only)."""
from qex_b200.kernel_timing import bytes_per_site, no_reuse_bytes_per_site


def test_compulsory_bytes_per_schur_call():
    # each link once per half sweep, each vector once; 12-real long links
    assert bytes_per_site(8, 0) == 2400 + 2448
    assert bytes_per_site(4, 0) == 1248 + 1296
    assert bytes_per_site(8, 2) == 512 + 536
    # 18-real long links below FP64 add 8 long links x 6 reals per sweep
    assert bytes_per_site(8, 1, recon12=False) == bytes_per_site(8, 1) + 2 * 4 * 2 * 24


def test_no_reuse_bytes_per_schur_call():
    # every neighbour's vector charged: fat+Naik FP64 3120 B and naive FP64
    # 1584 B per half sweep, plus the same-site operand of the second sweep
    assert no_reuse_bytes_per_site(8, 0) == 3120 + 3168
    assert no_reuse_bytes_per_site(4, 0) == 1584 + 1632
    assert no_reuse_bytes_per_site(8, 2) == bytes_per_site(8, 2) + 2 * 15 * 16
