"""Write tests/golden/tess_s58.npz: the TIME, PDCSAP_FLUX and PDCSAP_FLUX_ERR
columns and the RADIUS/LOGG header values of the TESS sector-58 2-minute
light curve that the reference bundles
(tess2022302161335-s0058-0000000021132157-0247-s_lc.fits, read by its
test1.py:86-95), read with this package's own FITS reader.  GPU boxes do not
have the reference tree; the fixture lets the tests run the reference's own
call on that light curve there.

    python tests/golden/make_tess_fixture.py [/path/to/reference]
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
NAME = "tess2022302161335-s0058-0000000021132157-0247-s_lc.fits"


def main(ref_root):
    from gtls_b200 import fits
    t, y, dy, hdr = fits.read_lightcurve(os.path.join(ref_root, NAME))
    np.savez_compressed(os.path.join(HERE, "tess_s58.npz"), time=t, pdcsap_flux=y, pdcsap_flux_err=dy,
                        radius=np.array(hdr["RADIUS"]), logg=np.array(hdr["LOGG"]))
    print("wrote", len(t), "rows")


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else os.environ.get("REFERENCE_ROOT", "/root/reference"))
