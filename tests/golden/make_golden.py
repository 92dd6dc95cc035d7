"""Copy the reference's numeric regression fixture into tests/golden/.

The reference ships exactly one numeric golden file,
utils/test/fig/reference/shearing/mri/history.txt: the history of its MRI
regression test (utils/test/test.py:974-990 with the defaults of
launchProblem, test.py:123-133): pro=mri, iso=1, 32x64x32 cells on
[-0.5,0.5]x[0,4]x[-0.5,0.5], Omega0=1e-3, ciso=1e-3, gamma=1.001, courant=0.8,
shearing-box x boundary, periodic y and z, HLLD/HLLD, MC slopes, FARGO off,
type='Test', beta=1000, amp=0, tlim=60000, dthist=100.

Run it once with the reference project's root as its argument
(python tests/golden/make_golden.py <reference root>); the copied file is
committed so the tests never read the reference at run time.
"""
import pathlib
import shutil
import sys

DST = pathlib.Path(__file__).with_name("mri_history_ref.txt")

if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: make_golden.py <reference project root>")
    src = pathlib.Path(sys.argv[1]) / "utils/test/fig/reference/shearing/mri/history.txt"
    shutil.copyfile(src, DST)
    print(f"wrote {DST} ({sum(1 for _ in open(DST)) - 1} rows)")
