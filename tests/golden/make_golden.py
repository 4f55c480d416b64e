"""Copies the reference's own regression fixtures (tomodir input files and
the recorded outputs that pin the forward / Jacobian / inner-solve path)
from a checkout of geophysics-ubonn/crtomo_stable into tests/golden/.

Run in an environment that has the reference checkout:
    python tests/golden/make_golden.py /path/to/crtomo_stable
The copied files are data (meshes, models, recorded voltages and inversion
logs); no reference source code is copied.
"""
import os
import shutil
import sys

HERE = os.path.dirname(os.path.abspath(__file__))

# case name -> (directory inside the reference's tests/, files relative to it)
CASES = {
    "minimal": ("minimal/Reference", [
        "grid/elem.dat", "grid/elec.dat", "rho/rho.dat", "mod/volt.dat", "exe/crmod.cfg",
        "exe/crtomo.cfg", "inv/volt00.dat", "inv/eps.ctr", "inv/inv.ctr", "inv/cjg.ctr",
        "inv/volt01.dat", "inv/volt02.dat", "inv/volt03.dat", "inv/coverage.mag", "inv/coverage.mag_fpi"]
        + [f"inv/rho{i:02d}.{e}" for i in range(4) for e in ("mag", "pha", "modl")]),
    "TestModInv": ("TestModInv/Reference", [
        "grid/elem.dat", "grid/elec.dat", "rho/rho.dat", "mod/volt.dat", "exe/crmod.cfg"]),
    "Lambda_search": ("Lambda_search/Test", [
        "grid/elem.dat", "grid/elec.dat", "rho/rho.dat", "mod/volt.dat", "exe/crmod.cfg",
        "exe/tmp.kfak"]),
    "mixed_surf": ("2.5D_mixed_surf/Reference", [
        "grid/elem.dat", "grid/elec.dat", "rho/rho.dat", "mod/volt.dat", "exe/crmod.cfg",
        "exe/crtomo.cfg", "inv/rho04.mag", "inv/rho04.pha", "inv/volt04.dat", "inv/coverage.mag"]),
    "non_ordered": ("non-ordered_boundary_conditions/Reference", [
        "grid/elem.dat", "grid/elec.dat", "rho/rho.dat", "mod/volt.dat", "exe/crmod.cfg",
        "exe/crtomo.cfg", "inv/rho04.mag", "inv/rho04.pha", "inv/volt04.dat", "inv/coverage.mag"]),
    "grid_decoupling": ("GridDecoupling/regular_grids/01_no_decoupling", [
        "grid/elem.dat", "grid/elec.dat", "rho/rho.dat", "mod/volt.dat", "exe/crmod.cfg",
        "config/config.dat"]),
    "dc_problem": ("DC_Problem/DC", [
        "grid/elem.dat", "grid/elec.dat", "mod/volt.dat", "exe/crtomo.cfg", "inv/eps.ctr",
        "inv/inv.ctr", "inv/volt00.dat"]),
    "dc_problem_complex": ("DC_Problem/Complex", [
        "grid/elem.dat", "grid/elec.dat", "mod/volt.dat", "exe/crtomo.cfg", "inv/eps.ctr",
        "inv/inv.ctr", "inv/cjg.ctr", "inv/rho00.mag", "inv/rho01.mag", "inv/rho01.modl"]),
}


def main(ref_root: str) -> None:
    for name, (sub, files) in CASES.items():
        for f in files:
            src = os.path.join(ref_root, "tests", sub, f)
            dst = os.path.join(HERE, name, f)
            os.makedirs(os.path.dirname(dst), exist_ok=True)
            shutil.copyfile(src, dst)
    print("copied", sum(len(f) for _, f in CASES.values()), "files")


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else "/root/reference")
