"""The FITS light-curve reader (gtls_b200/fits.py) on a file written here
and, when GTLS_TESS_FITS names one, on a real TESS light-curve product (the
reference bundles one, its sector-58 2-min file)."""
import os

import numpy as np
import pytest


def _card(key, value, comment=""):
    if isinstance(value, bool):
        v = "%20s" % ("T" if value else "F")
    elif isinstance(value, str):
        v = "'%-8s'" % value.replace("'", "''")
    elif isinstance(value, float):
        v = "%20s" % repr(value)
    else:
        v = "%20d" % value
    c = "%-8s= %s" % (key, v)
    if comment:
        c += " / " + comment
    return c.ljust(80)[:80]


def _block(cards):
    text = "".join(cards) + "END".ljust(80)
    text += " " * (-len(text) % 2880)
    return text.encode("ascii")


def _write(path, cols, primary):
    names = list(cols)
    nrows = len(cols[names[0]])
    forms = {np.dtype(">f8"): "D", np.dtype(">f4"): "E", np.dtype(">i4"): "J", np.dtype(">i2"): "I"}
    arrs = [np.asarray(cols[k]).astype(np.asarray(cols[k]).dtype.newbyteorder(">")) for k in names]
    width = sum(a.dtype.itemsize for a in arrs)
    hdr0 = [_card("SIMPLE", True), _card("BITPIX", 8), _card("NAXIS", 0), _card("EXTEND", True)]
    hdr0 += [_card(k, v) for k, v in primary.items()]
    hdr1 = [_card("XTENSION", "BINTABLE"), _card("BITPIX", 8), _card("NAXIS", 2), _card("NAXIS1", width),
            _card("NAXIS2", nrows), _card("PCOUNT", 0), _card("GCOUNT", 1), _card("TFIELDS", len(names))]
    for k, (name, a) in enumerate(zip(names, arrs), 1):
        hdr1 += [_card("TTYPE%d" % k, name), _card("TFORM%d" % k, "1" + forms[a.dtype])]
    rows = np.empty(nrows, dtype=[(n, a.dtype) for n, a in zip(names, arrs)])
    for n, a in zip(names, arrs):
        rows[n] = a
    data = rows.tobytes()
    data += b"\0" * (-len(data) % 2880)
    with open(path, "wb") as f:
        f.write(_block(hdr0) + _block(hdr1) + data)


def test_reader_round_trip(tmp_path):
    from gtls_b200 import fits
    rng = np.random.default_rng(1)
    n = 1234
    t = np.sort(rng.uniform(1000.0, 1027.0, n))
    y = 1.0 + rng.normal(0, 1e-3, n)
    y[5] = np.nan
    dy = rng.uniform(1e-4, 2e-4, n).astype(np.float32)
    q = rng.integers(0, 100, n).astype(np.int32)
    path = str(tmp_path / "lc.fits")
    _write(path, {"TIME": t, "PDCSAP_FLUX": y, "PDCSAP_FLUX_ERR": dy, "QUALITY": q},
           {"RADIUS": 0.87, "LOGG": 4.51, "OBJECT": "it's a test"})
    tt, yy, ee, hdr = fits.read_lightcurve(path)
    np.testing.assert_array_equal(tt, t)
    np.testing.assert_array_equal(yy, y)
    np.testing.assert_array_equal(ee, dy.astype(np.float64))
    assert hdr["RADIUS"] == 0.87 and hdr["LOGG"] == 4.51 and hdr["OBJECT"] == "it's a test"
    table = fits.read_table(*fits.read_hdus(path)[1])
    np.testing.assert_array_equal(table["QUALITY"], q)
    with pytest.raises(KeyError):
        fits.read_lightcurve(path, flux_col="SAP_FLUX")


def test_reads_a_tess_light_curve_file():
    path = os.environ.get("GTLS_TESS_FITS", "")
    if not os.path.exists(path):
        pytest.skip("GTLS_TESS_FITS does not name a TESS light-curve file")
    from gtls_b200 import fits, validate
    t, y, dy, hdr = fits.read_lightcurve(path)
    assert len(t) == len(y) == len(dy) > 19000
    assert "RADIUS" in hdr and "LOGG" in hdr
    ok = np.isfinite(t)
    assert np.all(np.diff(t[ok]) > 0) and 20.0 < np.ptp(t[ok]) < 30.0
    t, y, dy = validate.validate_inputs(t, y / np.nanmean(y), dy)
    assert len(t) > 15000
