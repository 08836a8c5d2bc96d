"""Copy the reference's own regression fixtures for the Green-function path.

The reference tests this path only through example runs compared against
``results_correct`` files (its CI: .gitlab-ci.yml, jobs Fe_bulk, Fe_bulk:susc,
graphene_pz, nanoribbon, Nb_100_Monolayer:ldos).  This script copies those example input decks and golden
outputs, unchanged, into ``tests/golden/<example>/`` so the tests can run
without the reference tree.  Run it from the repository root:

    python tests/golden/make_fixtures.py /path/to/reference
"""
import os
import shutil
import sys

FILES = {
    "Fe_bulk_susc": [
        "input", "basis", "Fe",
        "results_correct/scResult",
        "results_correct/TSOC/selfconsistency/selfconsistency_1Sites_dfttype=S_parts=2_norb=9_nkpt=1000_eta=1.0E-03.dat",
        "results_correct/TSOC/1Sites/HF/chihf_1_1_parts=2_parts3=1_norb=9_nkpt=1000_eta=1.0E-03.dat",
        "results_correct/TSOC/1Sites/RPA/chi_1_1_parts=2_parts3=1_norb=9_nkpt=1000_eta=1.0E-03.dat",
    ],
    "graphene": [
        "input", "basis", "Gr",
        "results_correct/scResult",
    ],
    "nanoribbon": [
        "input", "basis", "A2", "A3",
        "results_correct/scResult",
    ],
    "Nb_100_Monolayer": [
        "input", "basis", "Nb",
        "results_correct/scResult",
        "results_correct/TSOC/selfconsistency/selfconsistency_1Sites_dfttype=S_parts=2_norb=9_nkpt=1024_eta=1.0E-03_ev.dat",
        "results_correct/TSOC/1Sites/LDOS/ldosu_site=1_norb=9_nkpt=1024_eta=1.0E-03_ev.dat",
        "results_correct/TSOC/1Sites/LDOS/ldosd_site=1_norb=9_nkpt=1024_eta=1.0E-03_ev.dat",
        "results_correct/TSOC/1Sites/LDOS/lmdosu_site=1_norb=9_nkpt=1024_eta=1.0E-03_ev.dat",
        "results_correct/TSOC/1Sites/LDOS/lmdosd_site=1_norb=9_nkpt=1024_eta=1.0E-03_ev.dat",
    ],
}
NANO_SUFFIX = "parts=2_parts3=1_norb=2_nkpt=1000_eta=1.0E-03_ev_fixEf_Ef=-0.25_SOC=0.10_Vab=0.15_pxpy.dat"

# golden files are stored flat under short names
SHORT = {
    "results_correct/scResult": "scResult",
    "results_correct/TSOC/selfconsistency/selfconsistency_1Sites_dfttype=S_parts=2_norb=9_nkpt=1000_eta=1.0E-03.dat": "selfconsistency.dat",
    "results_correct/TSOC/1Sites/HF/chihf_1_1_parts=2_parts3=1_norb=9_nkpt=1000_eta=1.0E-03.dat": "chihf_1_1.dat",
    "results_correct/TSOC/1Sites/RPA/chi_1_1_parts=2_parts3=1_norb=9_nkpt=1000_eta=1.0E-03.dat": "chi_1_1.dat",
    "results_correct/TSOC/selfconsistency/selfconsistency_1Sites_dfttype=S_parts=2_norb=9_nkpt=1024_eta=1.0E-03_ev.dat":
        "selfconsistency.dat",
    "results_correct/TSOC/1Sites/LDOS/ldosu_site=1_norb=9_nkpt=1024_eta=1.0E-03_ev.dat": "ldosu_site=1.dat",
    "results_correct/TSOC/1Sites/LDOS/ldosd_site=1_norb=9_nkpt=1024_eta=1.0E-03_ev.dat": "ldosd_site=1.dat",
    "results_correct/TSOC/1Sites/LDOS/lmdosu_site=1_norb=9_nkpt=1024_eta=1.0E-03_ev.dat": "lmdosu_site=1.dat",
    "results_correct/TSOC/1Sites/LDOS/lmdosd_site=1_norb=9_nkpt=1024_eta=1.0E-03_ev.dat": "lmdosd_site=1.dat",
}


def main(ref_root: str) -> None:
    here = os.path.dirname(os.path.abspath(__file__))
    for ex, files in FILES.items():
        dst = os.path.join(here, ex)
        os.makedirs(dst, exist_ok=True)
        for f in files:
            src = os.path.join(ref_root, "examples", ex, f)
            shutil.copyfile(src, os.path.join(dst, SHORT.get(f, os.path.basename(f))))
        # nanoribbon: the self-consistent state and the 10 x 10 site pairs of chi_HF / chi_RPA
        if ex == "nanoribbon":
            base = os.path.join(ref_root, "examples", ex, "results_correct", "TSOC")
            sc = "selfconsistency_10Sites_dfttype=S_" + NANO_SUFFIX.replace("parts3=1_", "")
            shutil.copyfile(os.path.join(base, "selfconsistency", sc),
                            os.path.join(dst, "selfconsistency.dat"))
            for i in range(1, 11):
                for j in range(1, 11):
                    shutil.copyfile(os.path.join(base, "10Sites", "HF", f"chihf_{i}_{j}_" + NANO_SUFFIX),
                                    os.path.join(dst, f"chihf_{i}_{j}.dat"))
                    shutil.copyfile(os.path.join(base, "10Sites", "RPA", f"chi_{i}_{j}_" + NANO_SUFFIX),
                                    os.path.join(dst, f"chi_{i}_{j}.dat"))
            # calculate_all responses: disturbances, torques and effective fields per site and total
            for folder in ("SD", "CD", "LD", "SOT", "Beff"):
                src_dir = os.path.join(base, "10Sites", folder)
                os.makedirs(os.path.join(dst, "resp"), exist_ok=True)
                for f in sorted(os.listdir(src_dir)):
                    short = f.split("_parts=")[0] + ".dat"
                    shutil.copyfile(os.path.join(src_dir, f), os.path.join(dst, "resp", short))
        # the bulk reference densities of Nb (Un != 0): initialrho file of the element
        if ex == "Nb_100_Monolayer":
            shutil.copyfile(os.path.join(ref_root, "examples", ex, "results_correct", "FSOC", "selfconsistency",
                                         "initialrho_Nb_dfttype=S_parts=2_norb=9_nkpt=1024_eta=1.0E-03_ev.dat"),
                            os.path.join(dst, "initialrho_Nb.dat"))
        # the graphene self-consistency file has a run-dependent name
        if ex == "graphene":
            sc_dir = os.path.join(ref_root, "examples", ex, "results_correct", "FSOC", "selfconsistency")
            if os.path.isdir(sc_dir):
                for f in sorted(os.listdir(sc_dir)):
                    if f.startswith("selfconsistency_"):
                        shutil.copyfile(os.path.join(sc_dir, f), os.path.join(dst, "selfconsistency.dat"))
                        break
    print("fixtures written to", here)


if __name__ == "__main__":
    root = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("TITAN_REFERENCE")
    if not root:
        sys.exit("usage: make_fixtures.py <TITAN source tree>  (or set TITAN_REFERENCE)")
    main(root)
