"""ORACLE (test infrastructure only): run the reference's own CUDA build.

The binaries oracle/_ref/ref_* are the reference's sources compiled where they
lie by `make -C oracle ref` (driver: oracle/ref_harness/ref_main.cu).  Each
run writes an input.txt with the reference's keys (inc/parser.h) into a
temporary case folder and calls the binary there.  Used by
tests/golden/make_golden.py (fixtures) and by bench.py's reference arm (the
reference's CUDA timing); never by the agal_b200 package.
"""
from __future__ import annotations

import os
import subprocess
import tempfile
from pathlib import Path

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent
REF_BIN = HERE / "_ref"

BASE_KEYS = dict(MAX_LEVELS_WALL=1, MAX_LEVELS_INTERIOR=1, N_LEVEL_START=0, L_c=1.0, L_fy=1.0, L_fz=1.0,
                 N_RESTART=0, PERIODIC_X=0, PERIODIC_Y=0, PERIODIC_Z=0, N_ITER_TOTAL=1000,
                 S_FORCE_TYPE=2, S_BC_TYPE=0, S_CRITERION=0, N_PROBE=0, N_PROBE_FORCE=0, N_PRINT_LEVELS=0,
                 N_PRINT_LEVELS_IMAGE=0, P_OUTPUT=100000)


def write_input(d: Path, keys: dict, out_dir: Path) -> None:
    kv = dict(BASE_KEYS)
    kv.update(keys)
    kv["P_DIR_NAME"] = str(out_dir) + "/"
    kv["I_DIR_NAME"] = str(d) + "/"
    lines = [f"{k} {v}" for k, v in kv.items()]
    (d / "input.txt").write_text("\n".join(lines) + "\n")


def run_ref(binary: str, keys: dict, steps: int, keep_mb: int, dump: Path | None, n_timed: int = 0,
            region: int = 0, skip_last_regrid: bool = False, sphere: tuple | None = None,
            restart: Path | None = None, uniform: Path | None = None, geometry_txt: str | None = None) -> str:
    exe = REF_BIN / binary
    if not exe.exists():
        raise FileNotFoundError(f"{exe} missing: run `make -C oracle ref` first")
    with tempfile.TemporaryDirectory() as td:
        td = Path(td)
        (td / "out").mkdir()
        write_input(td, keys, td / "out")
        if sphere is not None:
            from agal_b200.geometry import icosphere, write_stl_ascii
            (td / "geometry").mkdir()
            write_stl_ascii(td / "geometry" / keys["G_FILENAME"], icosphere(*sphere))
        if geometry_txt is not None:
            (td / "geometry.txt").write_text(geometry_txt)
        cmd = [str(exe), str(td) + "/", str(dump) if dump else "-", str(steps), str(keep_mb), str(n_timed)]

        def big_stack():
            # M_Init builds the padded root grid as a stack VLA
            # (mesh_init.cu:332): ~50 MB at 8192^2.
            import resource
            resource.setrlimit(resource.RLIMIT_STACK, (1 << 30, resource.RLIM_INFINITY))

        env = dict(os.environ, REF_REGION=str(region), REF_SKIP_LAST_REGRID="1" if skip_last_regrid else "0",
                   REF_GEOM="1" if (sphere is not None or geometry_txt is not None) else "0", REF_RESTART="1" if restart is not None else "0",
                   REF_UNIFORM="1" if uniform is not None else "0")
        r = subprocess.run(cmd, cwd=td, capture_output=True, text=True, timeout=900, preexec_fn=big_stack,
                           env=env)
        if r.returncode != 0:
            raise RuntimeError(f"{binary} failed ({r.returncode}):\n{r.stdout[-3000:]}\n{r.stderr[-3000:]}")
        if restart is not None:
            restart.write_bytes((td / "out" / "restart.bin").read_bytes())
        if uniform is not None:
            uniform.write_bytes((td / "out" / "out_direct.dat").read_bytes())
        return r.stdout
