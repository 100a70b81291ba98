"""Point-source runs from run files: ``scripts/run_point_source.jl`` on the GPU.

    python -m crysplight_b200.run_point_source crysplight_b200/runs/point_csitl_teflon.toml [more.toml ...]

Each run file goes through ``run_from_config`` (src/config.jl:72-79): the
photons are transported by the CUDA library, ``output/<tag>/light.h5`` and a
copy of the run file are written, and the reference's summary is printed.
"""
from __future__ import annotations

import argparse


def main(argv=None):
    ap = argparse.ArgumentParser(description="point-source runs (scripts/run_point_source.jl)")
    ap.add_argument("configs", nargs="+", help="run files (runs/<tag>.toml)")
    ap.add_argument("--device", type=int, default=0)
    args = ap.parse_args(argv)
    from .config import run_from_config
    from .transport import Engine
    eng = Engine(args.device)
    try:
        for path in args.configs:
            run_from_config(path, engine=eng)
    finally:
        eng.close()


if __name__ == "__main__":
    main()
