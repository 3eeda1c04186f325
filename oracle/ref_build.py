"""Recipe: compile the reference's own C sources into test oracles.

The reference configures everything through ``#define``s in
``src/parameters.h`` (every configuration is a recompile, ``src/makefile``).
For each profile below this script

1. copies ``<reference>/src/*.c|*.h`` into a temporary directory (the
   reference tree is read-only and ``#include "parameters.h"`` would always
   pick the copy next to the sources, so an out-of-tree ``-I`` cannot override
   it),
2. rewrites the profile's ``#define`` lines of that copy of ``parameters.h``,
3. compiles with the reference's own flags (``gcc -O2``, ``src/makefile:10``)
   plus ``-fPIC``, and links

   * ``oracle/_ref/<profile>/libref.so`` = the reference objects (minus
     ``main.c``) + ``oracle/ref_driver.c``, with ``collision_treatment``
     wrapped to log the resolution order;
   * ``oracle/_ref/<profile>/ncorpion`` = the full reference program
     (``main.c`` included), reading ``./init.txt`` and writing its output
     files into the working directory (``pth`` = ``"./"``);
   * ``oracle/_ref/<profile>/ncorpion_gpu`` (brute-force and mesh profiles) =
     the same program with its two integration drivers taken from
     ``ncorpion_b200/host/rk4_gpu.c`` on ``libncgpu.so`` (the drop-in build).

Only build outputs are written under ``oracle/_ref/`` (git-ignored); the
temporary copy is deleted.  The shipped prebuilt ``src/ncorpion`` is never
copied, read or run.

Usage: ``python oracle/ref_build.py [--src DIR] [profile ...]`` (``DIR`` defaults to
``$NCORPION_REF_SRC``).
"""
from __future__ import annotations

import argparse
import glob
import os
import re
import shutil
import subprocess
import sys
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "_ref")
# the reference's src/ directory: --src, else $NCORPION_REF_SRC, else where this
# build machine mounts the reference
DEFAULT_SRC = os.environ.get("NCORPION_REF_SRC", "/root/reference/src")

COMMON = {
    "write_to_files_bool": "0",
    "make_animation_bool": "0",
    "write_cartesian_bool": "0",
    "write_elliptic_bool": "0",
    "write_collisions_bool": "0",
    "central_mass_bool": "1",
    "reduce_to_COM_bool": "1",
    "random_initial_bool": "0",
    "initial_cartesian_bool": "1",
    "seed_bool": "1",
    "one_collision_only_bool": "0",
    "openGL_bool": "0",
    "resume_simulation_bool": "0",
    "viscoelastic_bool": "0",
    "J2_bool": "0",
    "central_tides_bool": "0",
    "inner_fluid_disk_bool": "0",
    "mutual_bool": "1",
    "brute_force_bool": "0",
    "falcON_bool": "0",
    "standard_tree_bool": "0",
    "mesh_bool": "0",
    "elastic_collision_bool": "0",
    "inelastic_collision_bool": "0",
    "instant_merger_bool": "0",
    "fragmentation_bool": "0",
    "G": "1.",
    "pert_mass": "0.",
    "disruption_threshold": "0.1",
    "high_dumping_threshold": "100.",
    "pth": '"./"',
    "softening_parameter": "0.",
    "t_init": "0.",
}

BF = dict(COMMON, brute_force_bool="1")
MESH = dict(COMMON, mesh_bool="1", collision_cube_min="4.4", how_many_neighbours="16.0",
            sma_min="0.5", sma_max="2.0", inclination_max="0.015")

PROFILES = {
    # brute-force gravity only (src/physics.c:174-202), softening 0 and 0.5
    "bf_grav_s0": dict(BF, collision_bool="0", N_max="70000", N_0="2000",
                       t_end="0.01", time_step="0.001"),
    "bf_grav_s05": dict(BF, collision_bool="0", softening_parameter="0.5", N_max="70000",
                        N_0="2000", t_end="0.01", time_step="0.001"),
    # falcON gravity only (src/ffm.c, Dehnen 2002; the reference's default module): expansion order 3,
    # theta_min 0.45, the parameters.h defaults
    "tree_grav": dict(COMMON, falcON_bool="1", collision_bool="0", N_max="70000", N_0="2000",
                      t_end="0.01", time_step="0.001"),
    # brute-force gravity + brute-force collisions, instant merger: N=2000, 200 steps
    "bf_merge": dict(BF, collision_bool="1", instant_merger_bool="1", N_max="4096", N_0="2000",
                     t_end="0.2", time_step="0.001", output_step="50",
                     write_to_files_bool="1", write_cartesian_bool="1",
                     write_collisions_bool="1"),
    "bf_elastic": dict(BF, collision_bool="1", elastic_collision_bool="1", N_max="4096",
                       N_0="2000", t_end="0.05", time_step="0.001"),
    "bf_inelastic": dict(BF, collision_bool="1", inelastic_collision_bool="1",
                         collision_parameter="1.5", N_max="4096", N_0="2000",
                         t_end="0.05", time_step="0.001"),
    # mesh search + mesh gravity, instant merger, small cube for tests
    "mesh_merge_s": dict(MESH, collision_bool="1", instant_merger_bool="1",
                         collision_cube_cells="256", N_max="70000", N_0="20000",
                         t_end="0.005", time_step="0.0005"),
    "mesh_inelastic_s": dict(MESH, collision_bool="1", inelastic_collision_bool="1",
                             collision_parameter="1.5", collision_cube_cells="256",
                             N_max="70000", N_0="20000", t_end="0.005", time_step="0.0005"),
    "mesh_grav_s": dict(MESH, collision_bool="0", collision_cube_cells="256", N_max="70000",
                        N_0="20000", t_end="0.005", time_step="0.0005"),
    # fragmentation model (src/physics.c:710-1040), default constants (N_tilde 15)
    "bf_frag": dict(BF, collision_bool="1", fragmentation_bool="1", N_max="16384", N_0="2000",
                    t_end="0.05", time_step="0.001"),
    "mesh_frag_s": dict(MESH, collision_bool="1", fragmentation_bool="1", collision_cube_cells="256",
                        N_max="70000", N_0="20000", t_end="0.005", time_step="0.0005"),
    # "up to 4 fragments": N_tilde 4 on the 2 x 2 lattice {0,1,0,1}
    "mesh_frag4_s": dict(MESH, collision_bool="1", fragmentation_bool="1", collision_cube_cells="256",
                         N_tilde="4", pq_min_max="{0,1,0,1}", N_max="70000", N_0="20000",
                         t_end="0.005", time_step="0.0005"),
    # whole-program run of the mesh driver: 20,000 bodies, 100 steps, outputs every 25 steps
    "mesh_prog": dict(MESH, collision_bool="1", instant_merger_bool="1", collision_cube_cells="256",
                      N_max="30000", N_0="20000", t_end="0.05", time_step="0.0005", output_step="25",
                      write_to_files_bool="1", write_cartesian_bool="1", write_collisions_bool="1"),
    # the central body's J2 (src/physics.c:149-160): a constant J2_value, and
    # the fluid-body J2 (J2_value 0) that follows the central mass, with a
    # sideral period Tearth = 25 (J2 = 0.0316 for M = 1)
    "bf_grav_j2": dict(BF, collision_bool="0", softening_parameter="0.5", J2_bool="1", J2_value="0.0125",
                       N_max="70000", N_0="2000", t_end="0.01", time_step="0.001"),
    "bf_grav_j2f": dict(BF, collision_bool="0", J2_bool="1", J2_value="0.", Tearth="25.", N_max="70000",
                        N_0="2000", t_end="0.01", time_step="0.001"),
    "mesh_grav_j2f": dict(MESH, collision_bool="0", J2_bool="1", J2_value="0.", Tearth="25.",
                          collision_cube_cells="256", N_max="70000", N_0="20000", t_end="0.005",
                          time_step="0.0005"),
    # whole-program runs with J2: the brute-force and mesh drivers
    "bf_merge_j2": dict(BF, collision_bool="1", instant_merger_bool="1", J2_bool="1", J2_value="0.", Tearth="25.",
                        N_max="4096", N_0="2000", t_end="0.2", time_step="0.001", output_step="50",
                        write_to_files_bool="1", write_cartesian_bool="1", write_collisions_bool="1"),
    "mesh_prog_j2": dict(MESH, collision_bool="1", instant_merger_bool="1", J2_bool="1", J2_value="0.", Tearth="25.",
                         collision_cube_cells="256", N_max="30000", N_0="20000", t_end="0.05",
                         time_step="0.0005", output_step="25", write_to_files_bool="1",
                         write_cartesian_bool="1", write_collisions_bool="1"),
    # tides raised on the central body (src/physics.c:496-542) with a long time
    # lag (Delta_t = 1) so that every body changes SideralOmega; alone, and with
    # the fluid-body J2 that follows the changing rotation
    "bf_tides": dict(BF, collision_bool="0", softening_parameter="0.5", central_tides_bool="1", Delta_t="1.0",
                     N_max="70000", N_0="2000", t_end="0.01", time_step="0.001"),
    "bf_tides_j2f": dict(BF, collision_bool="0", central_tides_bool="1", Delta_t="1.0", J2_bool="1",
                         J2_value="0.", Tearth="25.", N_max="70000", N_0="2000", t_end="0.01", time_step="0.001"),
    "mesh_tides_j2f": dict(MESH, collision_bool="0", central_tides_bool="1", Delta_t="1.0", J2_bool="1",
                           J2_value="0.", Tearth="25.", collision_cube_cells="256", N_max="70000", N_0="20000",
                           t_end="0.005", time_step="0.0005"),
    # whole-program runs with tides and the fluid-body J2: both drivers
    "bf_merge_tides": dict(BF, collision_bool="1", instant_merger_bool="1", central_tides_bool="1", Delta_t="1.0",
                           J2_bool="1", J2_value="0.", Tearth="25.", N_max="4096", N_0="2000", t_end="0.2",
                           time_step="0.001", output_step="50", write_to_files_bool="1",
                           write_cartesian_bool="1", write_collisions_bool="1"),
    "mesh_prog_tides": dict(MESH, collision_bool="1", instant_merger_bool="1", central_tides_bool="1",
                            Delta_t="1.0", J2_bool="1", J2_value="0.", Tearth="25.", collision_cube_cells="256",
                            N_max="30000", N_0="20000", t_end="0.05", time_step="0.0005", output_step="25",
                            write_to_files_bool="1", write_cartesian_bool="1", write_collisions_bool="1"),
    # a larger run of the mesh driver (bench: whole-program wall time): 200,000
    # bodies of the mesh workload's disk, 20 steps, outputs every 10
    "mesh_prog_200k": dict(MESH, collision_bool="1", instant_merger_bool="1", collision_cube_cells="1024",
                           N_max="250000", N_0="200000", t_end="0.01", time_step="0.0005", output_step="10",
                           write_to_files_bool="1", write_cartesian_bool="1", write_collisions_bool="1"),
    # whole-program runs without output files, resuming files at the end (init.txt,
    # resume.txt): the final half backward drift / kick of both drivers; the mesh
    # driver also below switch_to_brute_force from the start (force_naive_bool)
    "bf_merge_resume": dict(BF, collision_bool="1", instant_merger_bool="1", N_max="4096", N_0="2000",
                            t_end="0.2", time_step="0.001", resume_simulation_bool="1"),
    "mesh_prog_resume": dict(MESH, collision_bool="1", instant_merger_bool="1", collision_cube_cells="256",
                             N_max="30000", N_0="20000", t_end="0.05", time_step="0.0005",
                             resume_simulation_bool="1"),
    "mesh_naive_resume": dict(MESH, collision_bool="1", instant_merger_bool="1", collision_cube_cells="256",
                              switch_to_brute_force="5000", N_max="4096", N_0="2000", t_end="0.05",
                              time_step="0.001", resume_simulation_bool="1"),
    # whole-program runs with the elliptic files (cart2ell, src/structure.c:172-284):
    # the brute-force driver with both coordinate sets and the fluid-body J2 (the
    # J2 correction of the semi-major axis), the mesh driver with elliptic files only
    "bf_merge_ell": dict(BF, collision_bool="1", instant_merger_bool="1", J2_bool="1", J2_value="0.", Tearth="25.",
                         N_max="4096", N_0="2000", t_end="0.2", time_step="0.001", output_step="50",
                         write_to_files_bool="1", write_cartesian_bool="1", write_elliptic_bool="1",
                         write_collisions_bool="1"),
    "mesh_prog_ell": dict(MESH, collision_bool="1", instant_merger_bool="1", collision_cube_cells="256",
                          N_max="30000", N_0="20000", t_end="0.05", time_step="0.0005", output_step="25",
                          write_to_files_bool="1", write_elliptic_bool="1", write_collisions_bool="1"),
    # the N = 1,048,576 mesh workload: 1024 cells per side (8.6 GB hash table)
    "mesh_merge_1m": dict(MESH, collision_bool="1", instant_merger_bool="1",
                          collision_cube_cells="1024", N_max="1100000", N_0="1048576",
                          t_end="0.05", time_step="0.0005"),
}

CFLAGS = ["-O2", "-fPIC", "-w"]


def write_params(src_params: str, dst_params: str, overrides: dict) -> None:
    with open(src_params) as f:
        lines = f.read().split("\n")
    seen = set()
    out = []
    for line in lines:
        m = re.match(r"^#define\s+(\w+)\s", line)
        if m and m.group(1) in overrides:
            name = m.group(1)
            out.append(f"#define {name} {overrides[name]}")
            seen.add(name)
        else:
            out.append(line)
    missing = set(overrides) - seen
    if missing:
        raise RuntimeError(f"parameters.h has no #define for {sorted(missing)}")
    with open(dst_params, "w") as f:
        f.write("\n".join(out))


def build(profile: str, src: str, verbose: bool = False) -> str:
    ov = PROFILES[profile]
    dst = os.path.join(OUT, profile)
    os.makedirs(dst, exist_ok=True)
    tmp = tempfile.mkdtemp(prefix=f"ncref_{profile}_")
    try:
        for p in glob.glob(os.path.join(src, "*.c")) + glob.glob(os.path.join(src, "*.h")):
            shutil.copy(p, tmp)
            os.chmod(os.path.join(tmp, os.path.basename(p)), 0o644)
        write_params(os.path.join(src, "parameters.h"), os.path.join(tmp, "parameters.h"), ov)
        shutil.copy(os.path.join(HERE, "ref_driver.c"), tmp)
        units = ["structure", "physics", "collision", "ffm", "rk4", "display", "spring"]
        objs = []
        for u in units + ["ref_driver"]:
            cmd = ["gcc", *CFLAGS, "-c", f"{u}.c", "-o", f"{u}.o"]
            subprocess.run(cmd, cwd=tmp, check=True)
            objs.append(f"{u}.o")
        lib = os.path.join(dst, "libref.so")
        subprocess.run(["gcc", "-shared", "-o", lib, *objs,
                        "-Wl,--wrap=collision_treatment", "-lm"], cwd=tmp, check=True)
        exe = os.path.join(dst, "ncorpion")
        subprocess.run(["gcc", *CFLAGS, "main.c", *[f"{u}.o" for u in units], "-lm", "-o", exe],
                       cwd=tmp, check=True)
        if ov.get("brute_force_bool") == "1" or ov.get("mesh_bool") == "1":
            build_dropin(tmp, dst, units)
        with open(os.path.join(dst, "profile.txt"), "w") as f:
            for k in sorted(ov):
                f.write(f"{k} {ov[k]}\n")
        if verbose:
            print(f"built {profile} -> {dst}")
        return dst
    finally:
        shutil.rmtree(tmp, ignore_errors=True)


def stale(profile: str) -> bool:
    """True when the profile is missing, its library predates ref_driver.c, or
    its drop-in program predates the C ABI header or the drop-in driver it was
    compiled from."""
    dst = os.path.join(OUT, profile)
    lib = os.path.join(dst, "libref.so")
    if not os.path.exists(lib) or os.path.getmtime(os.path.join(HERE, "ref_driver.c")) > os.path.getmtime(lib):
        return True
    ov = PROFILES[profile]
    if ov.get("brute_force_bool") == "1" or ov.get("mesh_bool") == "1":
        exe = os.path.join(dst, "ncorpion_gpu")
        root = os.path.dirname(HERE)
        deps = [os.path.join(root, "include", "ncgpu.h"), os.path.join(root, "ncorpion_b200", "host", "rk4_gpu.c")]
        if not os.path.exists(exe) or any(os.path.getmtime(d) > os.path.getmtime(exe) for d in deps):
            return True
    return False


def build_dropin(tmp: str, dst: str, units) -> None:
    """The reference program with its brute-force and mesh integrations
    replaced by ncorpion_b200/host/rk4_gpu.c on libncgpu.so: main.c is
    compiled with its two dispatch calls redirected, every other object is the
    reference's own."""
    root = os.path.dirname(HERE)
    pkg = os.path.join(root, "ncorpion_b200")
    lib = os.path.join(pkg, "libncgpu.so")
    if not os.path.exists(lib):
        raise RuntimeError("build libncgpu.so first (python -m ncorpion_b200.build)")
    redirect = ["-Dintegration_brute_force_SABA1=ncgpu_integration_brute_force_SABA1",
                "-Dintegration_mesh=ncgpu_integration_mesh"]
    subprocess.run(["gcc", *CFLAGS, *redirect, "-c", "main.c", "-o", "main_gpu.o"], cwd=tmp, check=True)
    subprocess.run(["gcc", *CFLAGS, "-I", tmp, "-I", os.path.join(root, "include"), "-c",
                    os.path.join(pkg, "host", "rk4_gpu.c"), "-o", "rk4_gpu.o"], cwd=tmp, check=True)
    rel = os.path.relpath(pkg, dst)
    subprocess.run(["gcc", "main_gpu.o", "rk4_gpu.o", *[f"{u}.o" for u in units], "-L", pkg, "-lncgpu",
                    f"-Wl,-rpath,$ORIGIN/{rel}", "-lm", "-o", os.path.join(dst, "ncorpion_gpu")],
                   cwd=tmp, check=True)


def main(argv=None) -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--src", default=DEFAULT_SRC)
    ap.add_argument("profiles", nargs="*")
    a = ap.parse_args(argv)
    if not os.path.isdir(a.src):
        print(f"reference sources not found at {a.src}; nothing built", file=sys.stderr)
        return 0
    for p in a.profiles or sorted(PROFILES):
        build(p, a.src, verbose=True)
    return 0


if __name__ == "__main__":
    sys.exit(main())
