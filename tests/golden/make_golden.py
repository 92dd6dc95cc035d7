"""Copy the reference's numeric regression fixture into tests/golden/.

The reference ships exactly one numeric golden file,
utils/test/fig/reference/shearing/mri/history.txt: the history of its MRI
regression test (utils/test/test.py:974-990 with the defaults of
launchProblem, test.py:123-133): pro=mri, iso=1, 32x64x32 cells on
[-0.5,0.5]x[0,4]x[-0.5,0.5], Omega0=1e-3, ciso=1e-3, gamma=1.001, courant=0.8,
shearing-box x boundary, periodic y and z, HLLD/HLLD, MC slopes, FARGO off,
type='Test', beta=1000, amp=0, tlim=60000, dthist=100.

This script is run once in a checkout that has the reference next to it; the
copied file is committed so the tests never read the reference at run time.
"""
import pathlib
import shutil
import sys

SRC = pathlib.Path(sys.argv[1] if len(sys.argv) > 1 else "/root/reference") / \
    "utils/test/fig/reference/shearing/mri/history.txt"
DST = pathlib.Path(__file__).with_name("mri_history_ref.txt")

if __name__ == "__main__":
    shutil.copyfile(SRC, DST)
    print(f"wrote {DST} ({sum(1 for _ in open(DST)) - 1} rows)")
