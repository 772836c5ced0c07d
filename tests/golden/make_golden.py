"""Generate the golden fixtures under tests/golden/ from the reference tree.

Run once in a container that has the ESPResSo source tree, named by
$P3MX_REFERENCE:

    P3MX_REFERENCE=<ESPResSo tree> python tests/golden/make_golden.py

Sources (paths relative to the ESPResSo tree):
  * testsuite/python/data/coulomb_cloud_wall_system.data  (id pos q f)
    with the parameters and energy of testsuite/python/coulomb_cloud_wall.py:40-47
  * testsuite/python/data/coulomb_tuning_system.npz (coulomb_tuning.py:37-47)
  * testsuite/python/data/lj_system.dat (lj.py:28-47)
  * testsuite/python/data/coulomb_mixed_periodicity_system.data (id pos q f,
    forces from MMM2D) with the parameters and the MMM2D energy of
    testsuite/python/coulomb_mixed_periodicity.py:30-40, 84-121 (ELC)
  * testsuite/python/data/p3m_magnetostatics_{system,expected}.data (id pos
    dip; id force torque per unit prefactor) with the parameters, energy and
    tolerances of testsuite/python/dipolar_mdlc_p3m_scafacos_p2nfft.py:115-152
  * testsuite/python/data/mdlc_reference_data_{forces_torques,energy}.dat
    (id pos dip force torque; energy, per unit prefactor) with the DLC
    parameters of dipolar_mdlc_p3m_scafacos_p2nfft.py:55-95
  * known answers written in testsuite/python/electrostatic_interactions.py:81-124
    and testsuite/python/p3m_madelung.py:69-313 (parameters and constants,
    electric and magnetic)
  * values of the reference's own math headers (bspline.hpp, AS_erfc_part.hpp,
    p3m/math.hpp) evaluated through oracle/_ref/libref_math.so, which
    oracle/Makefile compiles from the reference tree in place.
"""
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF = os.environ.get("P3MX_REFERENCE", "")
DATA = os.path.join(REF, "testsuite", "python", "data")
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))


def main():
    if not REF or not os.path.isdir(DATA):
        sys.exit("make_golden.py: set P3MX_REFERENCE to the ESPResSo source tree "
                 f"(got {REF!r})")
    d = np.genfromtxt(os.path.join(DATA, "coulomb_cloud_wall_system.data"))
    np.savez_compressed(
        os.path.join(HERE, "coulomb_cloud_wall.npz"),
        pos=d[:, 1:4], q=d[:, 4], forces=d[:, 5:8],
        box=np.array([10., 10., 10.]), mesh=np.array([64, 64, 64]), cao=7,
        alpha=2.70746, r_cut=1.001, accuracy=1e-3, energy=148.94229549,
        force_atol=2e-3, energy_atol=1e-3)

    t = np.load(os.path.join(DATA, "coulomb_tuning_system.npz"))
    np.savez_compressed(os.path.join(HERE, "coulomb_tuning.npz"),
                        pos=t["pos"], q=t["charges"], forces=t["forces"],
                        box=np.array([10., 10., 10.]), accuracy=5e-4,
                        force_atol=2e-3)

    lj = np.loadtxt(os.path.join(DATA, "lj_system.dat"))
    np.savez_compressed(os.path.join(HERE, "lj_system.npz"),
                        pos=lj[:, 1:4], forces=lj[:, 4:7], box=10.7437,
                        eps=1.0, sig=1.0, cut=1.12246, skin=0.4,
                        shift=0.2499999999700293)

    mp = np.genfromtxt(os.path.join(DATA, "coulomb_mixed_periodicity_system.data"))
    np.savez_compressed(
        os.path.join(HERE, "coulomb_mixed_periodicity.npz"),
        pos=mp[:, 1:4], q=mp[:, 4], forces=mp[:, 5:8],
        box=np.array([10., 10., 12.]), mesh=np.array([42, 42, 50]), r_cut=3.0,
        accuracy=1e-6, max_pw_error=1e-6, gap_size=3.0, energy=216.640984711,
        force_atol=1e-5, energy_atol=1e-4)

    mg = np.genfromtxt(os.path.join(DATA, "p3m_magnetostatics_system.data"))
    mx = np.genfromtxt(os.path.join(DATA, "p3m_magnetostatics_expected.data"))
    np.savez_compressed(
        os.path.join(HERE, "p3m_magnetostatics.npz"),
        pos=mg[:, 1:4], dip=mg[:, 4:7], forces=mx[:, 1:4], torques=mx[:, 4:7],
        box=float(np.cbrt(4 * 1000 * np.pi / (3 * 0.09))), prefactor=1.1, mesh=32,
        accuracy=1e-6, energy=5.570, force_tol=2e-3, torque_tol=2e-3, energy_tol=1e-3)

    md = np.genfromtxt(os.path.join(DATA, "mdlc_reference_data_forces_torques.dat"))
    me = float(np.genfromtxt(os.path.join(DATA, "mdlc_reference_data_energy.dat")))
    np.savez_compressed(
        os.path.join(HERE, "mdlc_reference.npz"),
        pos=md[:, 1:4], dip=md[:, 4:7], forces=md[:, 7:10], torques=md[:, 10:13],
        energy=me, box=float(np.cbrt(4 * 100 * np.pi / (3 * 0.3)) * 0.5), gap_size=2.0,
        prefactor=1.1, mesh=32, accuracy=1e-4, max_pw_error=1e-5, energy_tol=1e-3,
        force_tol=2e-3, torque_tol=2e-3)

    known = {
        "two_charges": {
            "source": "testsuite/python/electrostatic_interactions.py:81-124",
            "box": 20.0, "pos": [[9.0, 2.0, 2.0], [11.0, 2.0, 2.0]],
            "q": [1.0, -1.0], "prefactor": 1.1, "mesh": 22, "cao": 7,
            "r_cut": 8.90625, "alpha": 0.387611049779351, "accuracy": 1e-7,
            "energy_per_prefactor": -0.501062398379,
            "force_x_per_prefactor": 0.248921612, "tol": 1e-5,
            "dipole_tol": 1e-10},
        "madelung_wire": {
            "source": "testsuite/python/p3m_madelung.py:202-234",
            "n_pairs": 64, "mesh": 32, "cao": 7, "r_cut": 14.0,
            "alpha": 0.27362958, "accuracy": 1e-8,
            "madelung": float(-2.0 * np.log(2.0)), "base": [0, 0, 1],
            "energy_rtol": 5e-7, "pressure_rtol": 1e-6},
        "madelung_sheet": {
            "source": "testsuite/python/p3m_madelung.py:236-277",
            "n_pairs": 24, "mesh": 48, "cao": 7, "r_cut": 22.0,
            "alpha": 0.179719, "accuracy": 1e-8,
            "madelung": -1.6155426267128247, "base": [1, 1, 0],
            "energy_rtol": 1e-7, "pressure_rtol": 5e-7,
            "elc": {"maxPWerror": 1e-6, "gap_size": 16.0}},
        "madelung_cube": {
            "source": "testsuite/python/p3m_madelung.py:279-313",
            "n_pairs": 6, "mesh": 72, "cao": 7, "r_cut": 5.6,
            "alpha": 0.8163977, "accuracy": 1e-9,
            "madelung": -1.74756459463318219, "base": [1, 1, 1],
            "energy_rtol": 1e-6, "pressure_rtol": 5e-6,
            "gpu_params": {"mesh": 42, "cao": 7, "r_cut": 5.5,
                           "alpha": 0.709017, "accuracy": 3e-7}},
    }
    # dipolar P3M: energy per dipole x spacing^3 / dipm^2 of the magnetic
    # wire / sheet / cube (testsuite/python/p3m_madelung.py:69-200)
    known["magnetic"] = {
        "source": "testsuite/python/p3m_madelung.py:69-200",
        "dipm": 1.05,
        "wire": {"n_part": 64, "spacing": 1.2, "mesh": 48, "cao": 6, "r_cut": 28.0,
                 "alpha": 0.137582516, "accuracy": 1e-9,
                 "parallel": "-2 zeta(3)", "antiparallel": "3/2 zeta(3)", "rtol": 2e-9},
        "sheet": {"n_part": 32, "spacing": 2.4, "mesh": 48, "cao": 7, "r_cut": 33.6,
                  "alpha": 0.1186918, "accuracy": 1e-9,
                  "parallel": -2.54944, "antiparallel": 3.01716, "rtol": 4e-6},
        "cube": {"n_part": 8, "spacing": 2.4, "mesh": 64, "cao": 7, "r_cut": 8.2,
                 "alpha": 0.5091135, "accuracy": 5e-8,
                 "parallel": -2.67679, "antiparallel": 4.84473,
                 "rtol": 1e-6, "rtol_antiparallel": 3e-4},
    }
    with open(os.path.join(HERE, "known_answers.json"), "w") as fh:
        json.dump(known, fh, indent=1)

    from oracle import oracle as O
    O.build()
    r = O.ref_math()
    if r is None:
        raise SystemExit("oracle/_ref/libref_math.so missing: reference tree absent")
    xs = np.linspace(-0.5, 0.5, 41)
    bs = np.zeros((8, 7, len(xs)))
    for order in range(1, 8):
        for i in range(order):
            for k, x in enumerate(xs):
                bs[order, i, k] = r.ref_bspline(order, i, float(x))
    ds = np.linspace(0.0, 6.0, 121)
    ase = np.array([r.ref_as_erfc_part(float(x)) for x in ds])
    ss = np.linspace(-1.0, 1.0, 201)
    sinc = np.array([r.ref_sinc(float(x)) for x in ss])
    meshes = np.array([16, 22, 32, 42, 64])
    cot = np.zeros((8, len(meshes), 64))
    for cao in range(1, 8):
        for mi, m in enumerate(meshes):
            for n in range(-m // 2, m // 2):
                cot[cao, mi, n + 32] = r.ref_cotangent_sum(cao, n, 1.0 / m)
    np.savez_compressed(os.path.join(HERE, "ref_math.npz"), bspline_x=xs,
                        bspline=bs, as_erfc_d=ds, as_erfc=ase, sinc_x=ss,
                        sinc=sinc, cot_meshes=meshes, cot=cot)
    print("golden fixtures written to", HERE)


if __name__ == "__main__":
    main()
