"""Writes tests/golden/double_pendulum/: the reference's scene file
(assets/double_pendulum/double_pendulum.json, copied unchanged) and
Link{1,2}_Pos.csv, the reference's
double-pendulum trajectory data (nexdynipc/assets/reference_data/
double_pendulum/Link{1,2}_Pos.csv, one header row then time, x, y, z)
restricted to t <= 1.51 s (just past the scene's 1.5 s max_time, so that
interpolation covers every sample time) and thinned to every 5th
row, in the same layout.  Point NEXDYNIPC_REFERENCE at a checkout of the
reference (the directory that holds assets/):
    NEXDYNIPC_REFERENCE=<checkout> python tests/golden/make_double_pendulum_reference.py"""
import os

REF_ROOT = os.environ.get("NEXDYNIPC_REFERENCE", "")
SRC = os.path.join(REF_ROOT, "assets", "reference_data", "double_pendulum")
DST = os.path.join(os.path.dirname(os.path.abspath(__file__)), "double_pendulum")


def main():
    if not REF_ROOT or not os.path.isdir(SRC):
        raise SystemExit("set NEXDYNIPC_REFERENCE to a reference checkout (assets/reference_data/double_pendulum)")
    os.makedirs(DST, exist_ok=True)
    for body in ("Link1", "Link2"):
        with open(os.path.join(SRC, f"{body}_Pos.csv")) as f:
            lines = f.read().splitlines()
        rows = [ln for k, ln in enumerate(lines[1:]) if k % 5 == 0 and float(ln.split(",")[0]) <= 1.51]
        with open(os.path.join(DST, f"{body}_Pos.csv"), "w") as f:
            f.write("\n".join([lines[0]] + rows) + "\n")
    scene = os.path.join(REF_ROOT, "assets", "double_pendulum", "double_pendulum.json")
    with open(scene, "rb") as f, open(os.path.join(DST, "double_pendulum.json"), "wb") as g:
        g.write(f.read())


if __name__ == "__main__":
    main()
