"""Generate the golden fixtures of tests/golden from the reference tree.

Run in a checkout where the reference source tree is available (path given
as the first argument).  Reads, never executes, the reference's data files:
  - laminar_test/blasius_solution.dat  (Blasius table, eta/f/f' rows)
  - transition_test/temporal_modes_inlet.dat (binary TS inflow modes: the
    header and a checksum of the payload are kept)
  - laminar_test/Mean_profile_Retheta1100_ny32_Ly0.40.dat and
    tests/Mean_profile_Retheta1100_ny192_Ly0.60.dat (inflow profiles of
    inflow flags 2 and 5: ny, U_inlet(ny+1), V_inlet(ny); decoded here with
    numpy in the byte order that makes the file size match)
and writes small JSON fixtures the CPU tests compare against.
"""
import hashlib
import json
import os
import struct
import sys

import numpy as np


def main(ref):
    out = os.path.dirname(os.path.abspath(__file__))
    with open(os.path.join(ref, "laminar_test", "blasius_solution.dat")) as f:
        toks = f.read().split()
    n = int(toks[0])
    v = np.array([float(t) for t in toks[1:1 + 3 * n]])
    eta, fv, df = v[:n], v[n:2 * n], v[2 * n:]
    idx = list(range(0, n, 25)) + [n - 1]
    json.dump({"source": "laminar_test/blasius_solution.dat", "n": n, "index": idx,
               "eta": [eta[i] for i in idx], "f": [fv[i] for i in idx], "df": [df[i] for i in idx]},
              open(os.path.join(out, "blasius_ref.json"), "w"), indent=1)
    p = os.path.join(ref, "transition_test", "temporal_modes_inlet.dat")
    raw = open(p, "rb").read()
    ny, nm, mm = struct.unpack("<3i", raw[:12])
    beta, omega = struct.unpack("<2d", raw[12:28])
    off = 28
    ymesh = np.frombuffer(raw, "<f8", ny, off); off += 8 * ny
    zm = np.frombuffer(raw, "<f8", nm, off); off += 8 * nm
    tm = np.frombuffer(raw, "<f8", mm, off); off += 8 * mm
    nq = ny * nm * mm
    q = np.frombuffer(raw, "<f8", 6 * nq, off)
    json.dump({"source": "transition_test/temporal_modes_inlet.dat", "bytes": len(raw),
               "sha256": hashlib.sha256(raw).hexdigest(), "ny_inlet": ny, "n_modes": nm, "m_modes": mm,
               "beta": beta, "omega": omega, "ymesh_first_last": [ymesh[0], ymesh[-1]],
               "zmode": zm.tolist(), "tmode": tm.tolist(),
               "q_abs_sum": [float(np.abs(q[i * nq:(i + 1) * nq]).sum()) for i in range(6)]},
              open(os.path.join(out, "temporal_modes_ref.json"), "w"), indent=1)


    profs = []
    for rel in ("laminar_test/Mean_profile_Retheta1100_ny32_Ly0.40.dat",
                "tests/Mean_profile_Retheta1100_ny192_Ly0.60.dat"):
        raw = open(os.path.join(ref, rel), "rb").read()
        for order in ("<", ">"):
            ny = struct.unpack(order + "i", raw[:4])[0]
            if 0 < ny < 1 << 24 and len(raw) == 4 + 8 * (2 * ny + 1):
                break
        else:
            raise ValueError(rel + ": not an inflow profile")
        d = np.frombuffer(raw, order + "f8", 2 * ny + 1, 4)
        profs.append({"source": rel, "bytes": len(raw), "sha256": hashlib.sha256(raw).hexdigest(),
                      "order": "little" if order == "<" else "big", "ny": ny,
                      "U_inlet": d[:ny + 1].tolist(), "V_inlet": d[ny + 1:].tolist()})
    json.dump(profs, open(os.path.join(out, "inflow_profiles_ref.json"), "w"), indent=0)


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else os.environ["BLGPU_REFERENCE_DIR"])
