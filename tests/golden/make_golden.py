"""Extract the golden fixtures used by the parity tests from the reference checkout.

Run with the path of a checkout of the reference:

    python tests/golden/make_golden.py REFERENCE_CHECKOUT

It writes, next to this script:
  model_survey_fingerprints.json  Hamiltonian fingerprints of the reference's model survey
                                  (tests/regression/model_survey_reference.json) for the cases
                                  on the recursion path
  ex06_dos_fields.txt             examples/06_graphene_hbn_landau_levels/reference/dos_map.dat:
                                  energy [eV] and the DOS [1/eV/atom] at m = 0, 2, 16, 64 flux quanta
  ex07_dos_twists.txt             examples/07_graphene_hbn_twist_series/reference/dos.dat:
                                  energy [eV] and the DOS at 0.00 and 0.61 degrees
The numbers are copied as printed by the reference's plot.py (6 significant digits).
"""
import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CASES = ["graphene", "graphene+NeighLevels1", "graphene+NeighLevels2", "graphene+NeighLevels3",
         "graphene+MagField1", "eff", "eff+MoireOffDiag", "eff+MoireOffDiagMidpoint", "eff+MoireTwisted",
         "eff+MoireAddSecondMoire", "eff+MoireAddSecondMoire+Midpoint", "eff+MoireAddSecondMoire+Twisted2",
         "eff+MoireSecondMoireRotateFirst_off", "tbg", "tbg+MagField1", "sys_MoireEncapsulatedBilayerMC",
         "sys_MoireEncapsulatedBilayerMC+MoirePotential", "sys_MoireEncapsulatedBilayerMC+MoireOffDiag"]


def main(ref):
    fp = json.load(open(os.path.join(ref, "tests/regression/model_survey_reference.json")))
    out = {k: fp[k]["fingerprint"] for k in CASES}
    json.dump(out, open(os.path.join(HERE, "model_survey_fingerprints.json"), "w"), indent=1, sort_keys=True)

    lines = open(os.path.join(ref, "examples/06_graphene_hbn_landau_levels/reference/dos_map.dat")).read().split("\n")
    fields = lines[0].split()[2:]
    keep = [0, 1, 8, 32]  # columns of m = 0, 2, 16, 64
    with open(os.path.join(HERE, "ex06_dos_fields.txt"), "w") as f:
        f.write("# m 0 2 16 64 ; B[T] " + " ".join(fields[k] for k in keep) + "\n")
        for line in lines[1:]:
            if line.strip():
                v = line.split()
                f.write(" ".join([v[0]] + [v[1 + k] for k in keep]) + "\n")

    lines = open(os.path.join(ref, "examples/07_graphene_hbn_twist_series/reference/dos.dat")).read().split("\n")
    with open(os.path.join(HERE, "ex07_dos_twists.txt"), "w") as f:
        f.write("# twist[deg] 0.00 0.61\n")
        for line in lines[1:]:
            if line.strip():
                v = line.split()
                f.write(" ".join(v[:3]) + "\n")


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python tests/golden/make_golden.py REFERENCE_CHECKOUT")
    main(sys.argv[1])
