"""``python -m cfd_cavity_b200 [OPTIONS]``: runs the driver binary
``cavity_les`` (the reference binary's command line and run loops over the
CUDA library), building it in-tree first if it is missing."""
import os
import sys

from . import build


def main() -> None:
    exe = build.DRIVER
    if not os.path.exists(exe):
        build.build()
    os.execv(exe, [exe, *sys.argv[1:]])


if __name__ == "__main__":
    main()
