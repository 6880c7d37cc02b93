"""Reader of the reference's binary profile database (c2_db2bin_read).

Profiles are written in the COMER text format, turned into a binary
database by the reference's own makedb and db2bin (built from its sources by
oracle/build_ref.sh), and read back by this library.  The values must be
those of the text profiles as the reference's text reader converts them
(comer2_b200.textfmt.read_profiles): exact for target probabilities, context
vectors and their priors and norms, backgrounds and ENOs; transitions within
1e-7 (log computed in float or double); SS probabilities within 1.5e-4 (one
text quantum: makedb's reader and the query-side reader round them
differently).  Skipped where the reference tools are not built.
"""
import os
import subprocess

import numpy as np
import pytest

from comer2_b200 import synth as S
from comer2_b200 import textfmt

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF = os.path.join(ROOT, "oracle", "_ref")

needs_ref = pytest.mark.skipif(not (os.path.exists(os.path.join(REF, "makedb")) and
                                    os.path.exists(os.path.join(REF, "db2bin"))),
                               reason="reference tools not built (oracle/build_ref.sh)")


def _make_db(tmp, ps):
    pro = tmp / "pro"
    pro.mkdir()
    texts = []
    for k in range(ps.nprofiles):
        f = pro / ("p%04d.pro" % k)
        with open(f, "w") as fh:
            textfmt.write_profile(fh, ps, k, "p%04d" % k, "p%04d" % k)
        texts.append(f.read_text())
    opts = os.path.join(REF, "var", "options.txt")
    subprocess.run([os.path.join(REF, "makedb"), "-o", str(tmp / "db"), "-p", opts, "-d", str(pro)], check=True,
                   capture_output=True)
    subprocess.run([os.path.join(REF, "db2bin"), "-d", str(tmp / "db"), "-p", opts], check=True,
                   capture_output=True)
    return str(tmp / "db.bin"), textfmt.read_profiles("".join(texts))


@needs_ref
def test_db2bin_matches_text_profiles(tmp_path):
    from comer2_b200.native import read_db2bin
    rng = np.random.default_rng(5)
    q = S.random_profiles(rng, [80])
    ps = S.concat([S.random_profiles(rng, [31, 1, 140]), S.planted_homolog(rng, q, 90, 30, 60),
                   S.random_profiles(rng, [64, 7])])
    path, T = _make_db(tmp_path, ps)
    P = read_db2bin(path)
    assert P.nprofiles == T.nprofiles
    assert int(P.lengths.sum()) == int(T.lengths.sum())
    used = set()
    for k in range(P.nprofiles):
        L, o = int(P.lengths[k]), int(P.offsets[k])
        m = [t for t in range(T.nprofiles) if t not in used and T.lengths[t] == L and
             (T.aa[T.offsets[t]:T.offsets[t] + L] == P.aa[o:o + L]).all()][0]
        used.add(m)
        to = int(T.offsets[m])
        for f in ("trg", "cv", "cvprior", "cvnorm2"):
            assert np.array_equal(getattr(P, f)[o:o + L], getattr(T, f)[to:to + L]), f
        assert np.array_equal(P.bkg[k], T.bkg[m])
        assert P.eno[k] == pytest.approx(T.eno[m], abs=1e-6)
        assert np.allclose(P.trn[o + k:o + k + L + 1], T.trn[to + m:to + m + L + 1], rtol=1e-6, atol=1e-7)
        assert np.abs(P.ss[o:o + L] - T.ss[to:to + L]).max() <= 1.5e-4
        sp = P.ssstate[o:o + L]
        assert (np.where(sp == ord(" "), ord("C"), sp) == T.ssstate[to:to + L]).all()


def test_db2bin_rejects_other_files(tmp_path):
    from comer2_b200.native import C2Error, read_db2bin
    f = tmp_path / "x.bin"
    f.write_bytes(b"not a database" * 10)
    with pytest.raises(C2Error, match="not a COMER binary profile database"):
        read_db2bin(str(f))


@needs_ref
def test_db2bin_truncated_and_corrupt_files(tmp_path):
    """A database cut short anywhere, or with a corrupt count, address or
    profile length, is refused with an error message; nothing is read or
    sized beyond the file."""
    import struct
    from comer2_b200.native import C2Error, read_db2bin
    rng = np.random.default_rng(6)
    ps = S.random_profiles(rng, [31, 12, 140, 64])
    path, _ = _make_db(tmp_path, ps)
    data = open(path, "rb").read()
    hdr = len(b"COMER profile bin database v2.2")
    bad = tmp_path / "bad.bin"
    cuts = sorted({hdr - 3, hdr + 4, hdr + 16 + 8 * 40, len(data) // 3, len(data) // 2, len(data) - 300,
                   len(data) - 1})
    for cut in cuts:
        bad.write_bytes(data[:cut])
        with pytest.raises(C2Error, match="truncated|not a COMER"):
            read_db2bin(str(bad))
    # number of positions far beyond the file
    b = bytearray(data)
    b[hdr + 8:hdr + 16] = struct.pack("<Q", 1 << 60)
    bad.write_bytes(bytes(b))
    with pytest.raises(C2Error, match="number of positions"):
        read_db2bin(str(bad))
    # a section address past the end of the file
    b = bytearray(data)
    b[hdr + 16 + 8 * 30:hdr + 16 + 8 * 31] = struct.pack("<Q", len(data) + 4096)
    bad.write_bytes(bytes(b))
    with pytest.raises(C2Error, match="section address"):
        read_db2bin(str(bad))
    # a profile length that breaks the sum of lengths
    b = bytearray(data)
    a0 = struct.unpack("<Q", b[hdr + 16:hdr + 24])[0]
    b[a0:a0 + 4] = struct.pack("<i", 5)
    bad.write_bytes(bytes(b))
    with pytest.raises(C2Error, match="sum of profile lengths"):
        read_db2bin(str(bad))
    # the intact file still reads, descriptions included (in the database's
    # profile order, which makedb chooses)
    from comer2_b200.native import read_db2bin_descriptions
    assert read_db2bin(path).nprofiles == 4
    assert sorted(read_db2bin_descriptions(path)) == ["p%04d" % k for k in range(4)]


@needs_ref
def test_db2bin_range_reads_concatenate_to_the_whole(tmp_path):
    """Profile ranges read with c2_db2bin_read_range, concatenated, give the
    whole database field by field, transitions (one extra row per profile)
    included; ranges outside the database are refused."""
    from comer2_b200.native import C2Error, read_db2bin
    rng = np.random.default_rng(7)
    ps = S.random_profiles(rng, [31, 1, 140, 64, 7, 200, 2, 55])
    path, _ = _make_db(tmp_path, ps)
    W = read_db2bin(path)
    for cuts in ([0, 3, 8], [0, 1, 2, 5, 8], [0, 7, 8]):
        parts = [read_db2bin(path, a, b) for a, b in zip(cuts[:-1], cuts[1:])]
        for a, b, R in zip(cuts[:-1], cuts[1:], parts):
            assert np.array_equal(R.lengths, W.lengths[a:b])
            assert np.array_equal(R.offsets, W.offsets[a:b] - W.offsets[a])
        cat = S.concat(parts)
        for f in ("lengths", "offsets", "bkg", "eno", "trn", "trg", "cv", "cvprior", "cvnorm2", "ss", "ssstate",
                  "aa"):
            assert np.array_equal(getattr(cat, f), getattr(W, f)), f
    for a, b in ((-1, 2), (3, 3), (5, 2), (0, 9)):
        with pytest.raises(C2Error):
            read_db2bin(path, a, b)
