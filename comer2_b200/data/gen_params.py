"""Regenerate ``comer2_params.json`` from a COMER2 source tree.

The JSON holds the numbers of the reference install's parameter files, which
the search method depends on (GPL-3 data of the COMER2 project,
https://github.com/minmarg/comer2):

* ``src/env/comer.par``   -- Karlin-Altschul constants;
* ``src/env/options.txt`` -- default options, with ``SCOADJ`` forced to ``no``
  (the HDP score tables are not part of this implementation);
* ``src/env/ssss``        -- SS score table (raw triangular values);
* ``src/env/cvs2s``       -- CV score map (raw keys and scores; smoothing is
  applied at load time by ``comer2_b200.params.smooth_cvs2s``);
* the SS18 E-value model weights and adjustment constants, which the reference
  keeps as the array literal ``SSE_NN_WEIGHTS_`` in
  ``src/libmycu/cupro/CuDeviceMemory.cu:39-78``.

Usage: ``python gen_params.py <comer2-source-root>``.
"""
import json
import os
import re
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from comer2_b200 import params as P  # noqa: E402


def _nn_weights(src: str):
    m = re.search(r"SSE_NN_WEIGHTS_\[\]\s*=\s*\{(.*?)\};", src, re.S)
    if not m:
        raise SystemExit("SSE_NN_WEIGHTS_ not found")
    body = "\n".join(ln.split("//")[0] for ln in m.group(1).splitlines())
    return [float(t.rstrip("f")) for t in re.findall(r"-?\d+\.\d*f?", body)]


def main(root: str):
    env = os.path.join(root, "src", "env")
    rd = lambda p: open(os.path.join(env, p)).read()
    d = {
        "source": "COMER2 v2.03.03 parameter files (GPL-3 data), src/env and CuDeviceMemory.cu",
        "comer_par": P.parse_comer_par(rd("comer.par")),
        "options": P.parse_options(rd("options.txt")),
    }
    d["options"]["SCOADJ"] = "no"
    card, tri = P.parse_ssss(rd("ssss"))
    d["ssss"] = {"card": card, "tri": tri}
    keys, vals = P.parse_cvs2s(rd("cvs2s"))
    d["cvs2s"] = {"keys": keys, "values": vals}
    src = open(os.path.join(root, "src", "libmycu", "cupro", "CuDeviceMemory.cu")).read()
    d["sse_nn_weights"] = _nn_weights(src)
    out = os.path.join(HERE, "comer2_params.json")
    with open(out, "w") as fh:
        json.dump(d, fh, indent=1)
    print("wrote", out, "nn weights:", len(d["sse_nn_weights"]))


if __name__ == "__main__":
    root = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("COMER2_REFERENCE", "")
    if not root:
        sys.exit("usage: gen_params.py <reference-root>  (or set COMER2_REFERENCE)")
    main(root)
