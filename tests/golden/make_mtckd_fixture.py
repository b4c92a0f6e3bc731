"""Generate tests/golden/mtckd_h2o.npz from the reference's MT_CKD water
vapour continuum coefficient file (data/absco-ref_wv-mt-ckd.nc, read by
mt_ckd_h2o_module.f90:68-174), so that the continuum parity test runs on the
real coefficient table where the reference tree is absent.

The file's copyright notice (AER, MT_CKD 4.3) permits redistribution of the
data with the notice reproduced; it is stored in the fixture as `notice`.
Run in a checkout that has the LBLRTM data directory:
    python make_mtckd_fixture.py <lblrtm-data-dir>
"""
import os
import sys

import numpy as np
from scipy.io import netcdf_file


def main(data_dir):
    f = netcdf_file(os.path.join(data_dir, "absco-ref_wv-mt-ckd.nc"), "r", mmap=False)
    v = f.variables
    wn = np.array(v["wavenumbers"].data, dtype=np.float64)
    out = {
        "wavenumbers": wn,
        "self_absco_ref": np.array(v["self_absco_ref"].data, dtype=np.float64),
        "for_absco_ref": np.array(v["for_absco_ref"].data, dtype=np.float64),
        "self_texp": np.array(v["self_texp"].data, dtype=np.float64),
        "ref_press": np.float64(v["ref_press"].data),
        "ref_temp": np.float64(v["ref_temp"].data),
        "title": np.array(f._attributes["Title"].decode().strip()),
        "notice": np.array(f._attributes["Copyright"].decode().strip()),
    }
    assert np.allclose(np.diff(wn), wn[1] - wn[0])
    np.savez_compressed(os.path.join(os.path.dirname(os.path.abspath(__file__)), "mtckd_h2o.npz"),
                        **out)
    print(len(wn), "entries", out["title"])


if __name__ == "__main__":
    main(sys.argv[1])
