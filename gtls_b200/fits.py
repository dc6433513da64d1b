"""Light curves from FITS files (TESS/Kepler light-curve products).

The reference's scripts read light curves with astropy (test1.py:88-95:
``TIME``, ``PDCSAP_FLUX``, ``PDCSAP_FLUX_ERR`` of the first extension and
``RADIUS``/``LOGG`` of the primary header); astropy is not a dependency
here, so this module reads the FITS format itself: 2880-byte blocks of
80-character header cards, then the data of each HDU; binary-table
extensions (``XTENSION = 'BINTABLE'``) are decoded with NumPy from their
``TFORMn`` codes (big-endian), applying ``TSCALn``/``TZEROn`` to numeric
columns.  Only what light-curve files use is supported: no variable-length
arrays, no compressed images.
"""
import numpy as np

BLOCK = 2880
# TFORM code -> (numpy big-endian dtype, bytes per element)
_TFORM = {"L": ("i1", 1), "X": ("u1", 1), "B": ("u1", 1), "I": (">i2", 2), "J": (">i4", 4), "K": (">i8", 8),
          "A": ("S1", 1), "E": (">f4", 4), "D": (">f8", 8), "C": (">c8", 8), "M": (">c16", 16)}


def _parse_value(raw):
    raw = raw.strip()
    if raw.startswith("'"):
        end = raw.find("'", 1)
        while end != -1 and end + 1 < len(raw) and raw[end + 1] == "'":   # doubled quote inside a string
            end = raw.find("'", end + 2)
        return raw[1:end].replace("''", "'").rstrip()
    val = raw.split("/", 1)[0].strip()
    if val == "T":
        return True
    if val == "F":
        return False
    if val == "":
        return None
    try:
        return int(val)
    except ValueError:
        pass
    try:
        return float(val.replace("D", "E"))
    except ValueError:
        return val


def _read_header(buf, pos):
    """Header cards from byte ``pos``; returns (dict, position after the header)."""
    hdr = {}
    while True:
        if pos + BLOCK > len(buf):
            raise ValueError("FITS header runs past the end of the file")
        block = buf[pos:pos + BLOCK].decode("ascii", errors="replace")
        pos += BLOCK
        for i in range(0, BLOCK, 80):
            card = block[i:i + 80]
            key = card[:8].strip()
            if key == "END":
                return hdr, pos
            if card[8:10] == "= " and key:
                hdr[key] = _parse_value(card[10:])


def _data_size(hdr):
    naxis = int(hdr.get("NAXIS", 0))
    if naxis == 0:
        return 0
    n = 1
    for k in range(1, naxis + 1):
        n *= int(hdr["NAXIS%d" % k])
    n = abs(int(hdr.get("BITPIX", 8))) // 8 * int(hdr.get("GCOUNT", 1)) * (int(hdr.get("PCOUNT", 0)) + n)
    return n


def read_hdus(path):
    """Every HDU of a FITS file as (header dict, raw data bytes)."""
    with open(path, "rb") as f:
        buf = f.read()
    if not buf.startswith(b"SIMPLE  ="):
        raise ValueError("%s is not a FITS file" % path)
    hdus, pos = [], 0
    while pos + BLOCK <= len(buf):
        hdr, pos = _read_header(buf, pos)
        size = _data_size(hdr)
        hdus.append((hdr, buf[pos:pos + size]))
        pos += (size + BLOCK - 1) // BLOCK * BLOCK
    return hdus


def _columns(hdr):
    cols, off = [], 0
    for k in range(1, int(hdr["TFIELDS"]) + 1):
        form = str(hdr["TFORM%d" % k]).strip()
        i = 0
        while i < len(form) and form[i].isdigit():
            i += 1
        repeat = int(form[:i]) if i else 1
        code = form[i]
        if code not in _TFORM or code in ("P", "Q"):
            raise ValueError("unsupported TFORM %r" % form)
        dt, size = _TFORM[code]
        nbytes = (repeat + 7) // 8 if code == "X" else repeat * size
        cols.append(dict(name=str(hdr.get("TTYPE%d" % k, "COL%d" % k)).strip(), code=code, repeat=repeat, dtype=dt,
                         offset=off, nbytes=nbytes, scale=hdr.get("TSCAL%d" % k), zero=hdr.get("TZERO%d" % k)))
        off += nbytes
    if off != int(hdr["NAXIS1"]):
        raise ValueError("column widths do not add up to NAXIS1")
    return cols


def read_table(hdr, data):
    """A BINTABLE HDU as a dict of column name -> NumPy array (native byte order)."""
    if hdr.get("XTENSION") != "BINTABLE":
        raise ValueError("not a binary table extension")
    nrows, width = int(hdr["NAXIS2"]), int(hdr["NAXIS1"])
    raw = np.frombuffer(data[:nrows * width], dtype=np.uint8).reshape(nrows, width)
    out = {}
    for c in _columns(hdr):
        chunk = np.ascontiguousarray(raw[:, c["offset"]:c["offset"] + c["nbytes"]])
        if c["code"] == "A":
            arr = chunk.view("S%d" % c["repeat"]).reshape(nrows)
        elif c["code"] == "X":
            arr = chunk
        else:
            arr = chunk.view(c["dtype"]).reshape((nrows, c["repeat"]) if c["repeat"] > 1 else nrows)
            arr = arr.astype(arr.dtype.newbyteorder("="))
            if c["scale"] is not None or c["zero"] is not None:
                arr = arr * float(c["scale"] if c["scale"] is not None else 1.0) + \
                    float(c["zero"] if c["zero"] is not None else 0.0)
        out[c["name"]] = arr
    return out


def read_lightcurve(path, time_col="TIME", flux_col="PDCSAP_FLUX", err_col="PDCSAP_FLUX_ERR", ext=1):
    """(t, y, dy, primary header) of a light-curve file, as the reference's
    test1.py reads one: the columns of extension ``ext`` as float64 (NaNs
    kept; ``gtls(t, y, dy)`` drops them) and the primary header (``RADIUS``,
    ``LOGG``, ...)."""
    hdus = read_hdus(path)
    if ext >= len(hdus):
        raise ValueError("%s has no extension %d" % (path, ext))
    table = read_table(*hdus[ext])
    for c in (time_col, flux_col, err_col):
        if c is not None and c not in table:
            raise KeyError("column %s not in %s" % (c, sorted(table)))
    t = np.asarray(table[time_col], dtype=np.float64)
    y = np.asarray(table[flux_col], dtype=np.float64)
    dy = np.asarray(table[err_col], dtype=np.float64) if err_col is not None else None
    return t, y, dy, hdus[0][0]
