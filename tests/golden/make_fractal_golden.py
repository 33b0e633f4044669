"""Copy the reference's test/fractal golden vectors into a fixture.

    python tests/golden/make_fractal_golden.py [path/to/partmc/test/fractal]

Reads the two reference solutions that the reference's test_fractal_2.sh and
test_fractal_3.sh compare run_part against (column 1: dimensionless time,
column 2: dimensionless number concentration N/N0):
  ref_free_df_2_4_dimless_time_regrid.txt  free molecular regime, d_f = 2.4
  ref_cont_df_1_8_dimless_time_regrid.txt  continuum regime, d_f = 1.8
and writes them unchanged to tests/golden/fractal_ref.npz (arrays "free" and
"cont", each rows x 2), so the tests can run where the reference tree is not
present.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def main():
    src = sys.argv[1] if len(sys.argv) > 1 else "/root/reference/test/fractal"
    out = {}
    for key, name in (("free", "ref_free_df_2_4_dimless_time_regrid.txt"),
                      ("cont", "ref_cont_df_1_8_dimless_time_regrid.txt")):
        out[key] = np.loadtxt(os.path.join(src, name))
        assert out[key].ndim == 2 and out[key].shape[1] == 2
    np.savez(os.path.join(HERE, "fractal_ref.npz"), **out)
    print({k: v.shape for k, v in out.items()})


if __name__ == "__main__":
    main()
