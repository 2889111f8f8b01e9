"""Command-line runner: python -m fibrenet_b200.cli <input_file> [--device N] [--strict]

SimulationManager's Initialize + Run + Close on a reference input file, with
the input file and device given on the command line (FibreNet.cpp:6-15 asks
for them interactively)."""
import argparse
import sys

from . import files


def main(argv=None) -> int:
    p = argparse.ArgumentParser(prog="fibrenet_b200.cli")
    p.add_argument("input_file")
    p.add_argument("--device", type=int, default=0)
    p.add_argument("--strict", action="store_true", help="read every number as a double, etc.")
    a = p.parse_args(argv)
    try:
        files.run_input(a.input_file, a.device, a.strict)
    except files.InputError as e:
        print(f"fibrenet: {e}", file=sys.stderr)
        return 1
    return 0


if __name__ == "__main__":
    sys.exit(main())
