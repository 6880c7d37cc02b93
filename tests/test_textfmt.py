"""COMER text profile format: write and read back (CPU)."""
import io
import os
import subprocess

import numpy as np
import pytest

from comer2_b200 import synth as S, textfmt

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_roundtrip():
    rng = np.random.default_rng(3)
    ps = S.random_profiles(rng, [17, 40])
    buf = io.StringIO()
    for k in range(ps.nprofiles):
        textfmt.write_profile(buf, ps, k, "p%d" % k, "desc %d" % k)
    back = textfmt.read_profiles(buf.getvalue())
    assert back.nprofiles == 2 and list(back.lengths) == [17, 40]
    for name in ("trg", "trn", "cv", "cvprior", "cvnorm2", "ss", "bkg", "eno"):
        assert np.array_equal(getattr(back, name), getattr(ps, name)), name
    assert np.array_equal(back.aa, ps.aa) and np.array_equal(back.ssstate, ps.ssstate)


@pytest.mark.skipif(not os.path.exists(os.path.join(ROOT, "oracle", "_ref", "makedb")),
                    reason="reference tools not built (oracle/build_ref.sh)")
def test_reference_makedb_accepts(tmp_path):
    rng = np.random.default_rng(5)
    ps = S.random_profiles(rng, [30, 31])
    for k in range(2):
        with open(tmp_path / ("p%d.pro" % k), "w") as fh:
            textfmt.write_profile(fh, ps, k, "p%d" % k, "p%d" % k)
    ref = os.path.join(ROOT, "oracle", "_ref")
    opts = os.path.join(ref, "var", "options.txt")
    subprocess.run([os.path.join(ref, "makedb"), "-o", str(tmp_path / "db"), "-p", opts, "-d", str(tmp_path)],
                   check=True, capture_output=True)
    subprocess.run([os.path.join(ref, "db2bin"), "-d", str(tmp_path / "db"), "-p", opts], check=True,
                   capture_output=True)
    assert (tmp_path / "db.bin").stat().st_size > 0
