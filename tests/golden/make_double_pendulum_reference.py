"""Writes tests/golden/double_pendulum/Link{1,2}_Pos.csv: the reference's
double-pendulum trajectory data (nexdynipc/assets/reference_data/
double_pendulum/Link{1,2}_Pos.csv, one header row then time, x, y, z)
restricted to t <= 1.51 s (just past the scene's 1.5 s max_time, so that
interpolation covers every sample time) and thinned to every 5th
row, in the same layout.  Run in a checkout that has the reference at
/root/reference:  python tests/golden/make_double_pendulum_reference.py"""
import os

SRC = "/root/reference/assets/reference_data/double_pendulum"
DST = os.path.join(os.path.dirname(os.path.abspath(__file__)), "double_pendulum")


def main():
    os.makedirs(DST, exist_ok=True)
    for body in ("Link1", "Link2"):
        with open(os.path.join(SRC, f"{body}_Pos.csv")) as f:
            lines = f.read().splitlines()
        rows = [ln for k, ln in enumerate(lines[1:]) if k % 5 == 0 and float(ln.split(",")[0]) <= 1.51]
        with open(os.path.join(DST, f"{body}_Pos.csv"), "w") as f:
            f.write("\n".join([lines[0]] + rows) + "\n")


if __name__ == "__main__":
    main()
