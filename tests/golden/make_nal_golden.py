"""NAL container fixture from the reference's own stream_helper (src/utils/stream_helper.py).
Run here, where the reference sources exist:  python tests/golden/make_nal_golden.py"""
import io
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def sequence():
    """Units to write; payloads are regenerated from a seed (payload(i, n)) to keep this small."""
    units = []
    for h, w in [(1080, 1920), (720, 1280), (1080, 1920)]:
        units.append(("sps", h, w))
    for i, n in enumerate([0, 5, 127, 128, 16383, 16384, 70000]):
        units.append(("ip", i % 2 == 0, i % 3, (i * 9) % 64, i % 9, i % 2, n))
    return units


def payload(i, n):
    return np.random.default_rng(7700 + i).integers(0, 256, n).astype(np.uint8).tobytes()


def main(ref=None):
    ref = ref or os.environ.get("DCVC_REFERENCE")
    if not ref:
        raise SystemExit("set DCVC_REFERENCE to the reference checkout")
    sys.path.insert(0, ref)
    from src.utils import stream_helper as S
    f = io.BytesIO()
    helper = S.SPSHelper()
    written = []
    for i, u in enumerate(sequence()):
        if u[0] == "sps":
            sps = {"sps_id": -1, "height": u[1], "width": u[2]}
            sid, new = helper.get_sps_id(sps)
            sps["sps_id"] = sid
            written.append(["sps", sid, bool(new), S.write_sps(f, sps) if new else 0])
        else:
            _, is_i, sid, qp, ec, reset, n = u
            written.append(["ip", S.write_ip(f, is_i, sid, qp, ec, reset, payload(i, n))])
    import hashlib
    data = f.getvalue()
    with open(os.path.join(HERE, "nal_golden.json"), "w") as out:
        json.dump({"sequence": sequence(), "written": written, "size": len(data),
                   "sha256": hashlib.sha256(data).hexdigest(), "head": data[:64].hex()}, out)


if __name__ == "__main__":
    main()
