"""Pack the reference's published driver outputs into tests/golden/ref_published.npz
(run in the container that has the reference tree; commits only the .npz and
this script).

    python tests/golden/make_published.py

The reference ships, beside its driver main.cpp and config.toml, the csv files
that driver wrote (Test_Output/test_solution_<sig>.csv: 6 nodal points per
element, x y z 0 and the three DD components; Test_Output/test_stresses_<sig>.csv:
Sxx Syy Szz Sxy Sxz Syz at Test_Output/observation_points.csv), printed with the
C++ stream default of 6 significant digits, for five of its meshes
(Mesh_Files/{Elems,Nodes}_<mesh>_32.npy).  The settings are those of the shipped
config.toml (config.toml:72-133): fix_tip = 1, cp_offset = 0.125,
is_dd_local = false, S_zz = -1 (compression positive, so s_inf zz = +1),
Shear_modulus = 1, Poisson_ratio = 0.35.

Stored per case <sig> (psc_24, psc_121, psc_1025, elc_124, elc_550): the mesh
arrays exactly as shipped (dtype, shape and Fortran order), the solution and the
stresses; and the observation points (n x 3, as in the csv).
"""
import os
import sys

import numpy as np

REF = os.environ.get('HFPX_REFERENCE', '')
if not os.path.isdir(REF):
    sys.exit('set HFPX_REFERENCE to the reference tree')
HERE = os.path.dirname(os.path.abspath(__file__))

CASES = {'psc_24': 'pennymesh24el', 'psc_121': 'pennymesh121el', 'psc_1025': 'pennymesh1025el',
         'elc_124': 'elliptical_124_el', 'elc_550': 'elliptical_550_el'}


def main():
    out = {'pts': np.loadtxt(os.path.join(REF, 'Test_Output', 'observation_points.csv'), delimiter=',')}
    for sig, mesh in CASES.items():
        out[f'{sig}_conn'] = np.load(os.path.join(REF, 'Mesh_Files', f'Elems_{mesh}_32.npy'))
        out[f'{sig}_nods'] = np.load(os.path.join(REF, 'Mesh_Files', f'Nodes_{mesh}_32.npy'))
        for kind in ('solution', 'stresses'):
            out[f'{sig}_{kind}'] = np.loadtxt(
                os.path.join(REF, 'Test_Output', f'test_{kind}_{sig}_ele.csv'), delimiter=',')
    np.savez_compressed(os.path.join(HERE, 'ref_published.npz'), **out)


if __name__ == '__main__':
    main()
