"""Extracts the reference's printed per-step norms from its golden .output files
into reference_outputs.json.  Run once in a container where the reference
sources are mounted (read as text only); the JSON is the committed fixture:

    python tests/golden/make_golden.py <path of the reference checkout>
"""
import json
import os
import re
import sys

CASES = {
    # name: (relative path of the .output file, regex of the printed value)
    "advection_diffusion_vortex_mf": (
        "applications/mp-advec-diff/cases/tests/advection_diffusion_vortex_mf.mpirun=4.output",
        r"\|\| advected field \|\|L2 = ([0-9.eE+-]+)"),
    "advection_diffusion_vortex_mf_3d": (
        "applications/mp-advec-diff/cases/tests/advection_diffusion_vortex_mf_3d.mpirun=4.output",
        r"\|\| advected field \|\|L2 = ([0-9.eE+-]+)"),
    "advection_diffusion_vortex": (
        "applications/mp-advec-diff/cases/tests/advection_diffusion_vortex.mpirun=4.output",
        r"\|\| advected field \|\|L2 = ([0-9.eE+-]+)"),
    "advection_diffusion_vortex_mf_inflow_outflow_3d": (
        "applications/mp-advec-diff/cases/tests/advection_diffusion_vortex_mf_inflow_outflow_3d.mpirun=4.output",
        r"\|\| advected field \|\|L2 = ([0-9.eE+-]+)"),
    "advection_diffusion_vortex_mf_inflow_outflow": (
        "applications/mp-advec-diff/cases/tests/advection_diffusion_vortex_mf_inflow_outflow.mpirun=4.output",
        r"\|\| advected field \|\|L2 = ([0-9.eE+-]+)"),
    "advection_diffusion_vortex_mf_supg": (
        "applications/mp-advec-diff/cases/tests/advection_diffusion_vortex_mf_supg.mpirun=4.output",
        r"\|\| advected field \|\|L2 = ([0-9.eE+-]+)"),
    "unidirectional_heat_transfer": (
        "applications/mp-heat-transfer/cases/unidirectional_heat_transfer/tests/"
        "unidirectional_heat_transfer.mpirun=4.output",
        r"\|\|solution\|\| = ([0-9.eE+-]+)"),
    "unidirectional_heat_transfer_with_convection": (
        "applications/mp-heat-transfer/cases/unidirectional_heat_transfer/tests/"
        "unidirectional_heat_transfer_with_convection.mpirun=4.output",
        r"\|\|solution\|\| = ([0-9.eE+-]+)"),
    "unidirectional_heat_transfer_with_radiation": (
        "applications/mp-heat-transfer/cases/unidirectional_heat_transfer/tests/"
        "unidirectional_heat_transfer_with_radiation.mpirun=4.output",
        r"\|\|solution\|\| = ([0-9.eE+-]+)"),
    "unidirectional_heat_transfer_with_radiation_and_convection": (
        "applications/mp-heat-transfer/cases/unidirectional_heat_transfer/tests/"
        "unidirectional_heat_transfer_with_radiation_and_convection.mpirun=4.output",
        r"\|\|solution\|\| = ([0-9.eE+-]+)"),
    "unidirectional_heat_transfer_with_velocity": (
        "applications/mp-heat-transfer/cases/unidirectional_heat_transfer/tests/"
        "unidirectional_heat_transfer_with_velocity.mpirun=4.output",
        r"\|\|solution\|\| = ([0-9.eE+-]+)"),
    "unidirectional_heat_transfer_with_two_phase": (
        "applications/mp-heat-transfer/cases/unidirectional_heat_transfer/tests/"
        "unidirectional_heat_transfer_with_two_phase.mpirun=4.output",
        r"\|\|solution\|\| = ([0-9.eE+-]+)"),
    "unidirectional_heat_transfer_with_two_phase_rho_times_cp": (
        "applications/mp-heat-transfer/cases/unidirectional_heat_transfer/tests/"
        "unidirectional_heat_transfer_with_two_phase_rho_times_cp.mpirun=4.output",
        r"\|\|solution\|\| = ([0-9.eE+-]+)"),
    "unidirectional_heat_transfer_with_velocity_and_solidification": (
        "applications/mp-heat-transfer/cases/unidirectional_heat_transfer/tests/"
        "unidirectional_heat_transfer_with_velocity_and_solidification.mpirun=4.output",
        r"\|\|solution\|\| = ([0-9.eE+-]+)"),
    "unidirectional_heat_transfer_with_two_phase_and_solidification": (
        "applications/mp-heat-transfer/cases/unidirectional_heat_transfer/tests/"
        "unidirectional_heat_transfer_with_two_phase_and_solidification.mpirun=4.output",
        r"\|\|solution\|\| = ([0-9.eE+-]+)"),
}


def main(root):
    out = {}
    for name, (rel, pat) in CASES.items():
        text = open(os.path.join(root, rel)).read()
        vals = re.findall(pat, text)
        out[name] = {"source": rel, "printed": vals, "values": [float(v) for v in vals]}
    here = os.path.dirname(os.path.abspath(__file__))
    with open(os.path.join(here, "reference_outputs.json"), "w") as f:
        json.dump(out, f, indent=1)


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: make_golden.py <path of the reference checkout>")
    main(sys.argv[1])
