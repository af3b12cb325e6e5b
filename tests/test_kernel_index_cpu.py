"""Index arithmetic of the sweeps' kernels, restated on the CPU in the kernels'
own number types.  These formulas decide which shared-memory slot a lane reads
or writes; an error in them would drop or duplicate work, so they are checked
here over every shape the kernels accept:

* the reciprocal band's staging (typed_impl.cuh, k_recip_sweep): lanes run
  over the flat rows x (cols - 1) entries of a band of at most 20 rows and 64
  columns and take the row of entry e as floor((e + 1/2) * (1 / (cols - 1)))
  in f32;
* the reciprocal band's 32-bit entry address (BandSampler::entry): a texel at
  band column cx and row cy is read at base + 512 cy + 8 cx, formed as
  (base - 520 bits(2^23)) + (bits(2^23 + cy) << 9) + (bits(2^23 + cx) << 3)
  modulo 2^32;
* the depth sweep's row pairing for 16-wide tiles (k_sweep_tiled): the
  horizontal pass visits footprint rows through a map that must be a
  permutation, and that puts the two half-warps of a warp on rows d apart with
  d x PXp = 16 (mod 32) words wherever it pairs them.
"""
import numpy as np

BAND_PITCH, BAND_ROWS = 64, 20
TWO23 = np.float32(8388608.0)


def test_band_staging_rows_are_exact():
    for cols in range(2, BAND_PITCH + 1):
        c1 = cols - 1
        inv = np.float32(1.0) / np.float32(c1)
        for rows in range(1, BAND_ROWS + 1):
            e = np.arange(rows * c1, dtype=np.int64)
            rr = ((e.astype(np.float32) + np.float32(0.5)) * inv).astype(np.int64)
            assert np.array_equal(rr, e // c1), (rows, cols)
            c = e - rr * c1
            assert c.min() >= 0 and c.max() < c1


def test_band_entry_address_folds_the_shift():
    sb = int(TWO23.view(np.uint32))
    for base in (0, 1024, 47000, 227 * 1024 - BAND_ROWS * 512):
        cbase = (base - (8 + 8 * BAND_PITCH) * sb) % 2 ** 32
        for cy in range(BAND_ROWS):
            tv = int((TWO23 + np.float32(cy)).view(np.uint32))
            cx = np.arange(BAND_PITCH)
            tu = (TWO23 + cx.astype(np.float32)).view(np.uint32).astype(np.int64)
            addr = (cbase + ((tv << 9) % 2 ** 32) + ((tu << 3) % 2 ** 32)) % 2 ** 32
            assert np.array_equal(addr, base + 512 * cy + 8 * cx)


def row_map(py, pxp):
    """The map k_sweep_tiled builds for a 16-wide tile (rowmap)."""
    pd = 0
    for d in range(1, 32):
        if (d * pxp) % 32 == 16:
            pd = d
            break
    out = []
    for q in range(py):
        row = q
        if pd:
            blk = 2 * pd
            bq = q // blk
            if (bq + 1) * blk <= py:
                w = q - bq * blk
                row = bq * blk + (w >> 1) + (w & 1) * pd
        out.append(row)
    return out, pd


def test_sweep_row_pairing_is_a_permutation_with_disjoint_banks():
    tx = ty = 16
    for stride in range(1, 13):
        for window in (3, 5, 7, 9):
            px = (tx - 1) * stride + window
            py = (ty - 1) * stride + window
            pxs = (px + stride - 1) // stride
            pxp = pxs * stride
            rows, pd = row_map(py, pxp)
            assert sorted(rows) == list(range(py)), (stride, window)
            # a warp's outputs i .. i + 31 are the map's entries 2p and 2p + 1
            for p in range(py // 2):
                a, b = rows[2 * p], rows[2 * p + 1]
                if pd and abs(b - a) == pd:
                    banks_a = {(a * pxp + c) % 32 for c in range(16)}
                    banks_b = {(b * pxp + c) % 32 for c in range(16)}
                    assert not banks_a & banks_b


def test_contrast_gate_f32_error_bound():
    """k_recip_prepare decides the source contrast gate in f32 on the exact
    texels and fractions of the f64 taps whenever the f32 contrast lies more
    than M 2^-16 from the gate (M the largest texel magnitude read); the f32
    bilinear is within M 2^-20 of the f64 one, so the decision is the exact
    one.  Restated here with f32 products and sums rounded separately (a wider
    error than the kernel's FMAs) over texels of every storage scale."""
    rng = np.random.default_rng(7)
    for scale in (1.0, 255.0, 1e-3, 1e4):
        t = (rng.random((200000, 4)) * scale).astype(np.float32)
        frac = rng.random((200000, 2))
        tx, ty = frac[:, 0].astype(np.float32), frac[:, 1].astype(np.float32)
        v00, v10, v01, v11 = (t[:, i] for i in range(4))
        top = (v10 - v00) * tx + v00
        bot = (v11 - v01) * tx + v01
        f32 = ((bot - top) * ty + top).astype(np.float64)
        d = t.astype(np.float64)
        fx, fy = frac[:, 0], frac[:, 1]
        top64 = d[:, 0] * (1.0 - fx) + d[:, 1] * fx
        bot64 = d[:, 2] * (1.0 - fx) + d[:, 3] * fx
        f64 = top64 * (1.0 - fy) + bot64 * fy
        mag = np.abs(t).max(axis=1).astype(np.float64)
        assert np.all(np.abs(f32 - f64) <= mag * 2.0 ** -20), scale
