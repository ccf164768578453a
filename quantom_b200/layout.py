"""numpy views of the reference LIMA_MD data layout.

The C-ABI (include/lima_abi.h) takes arrays in the reference's own struct
layout so a caller holding the reference's Box arrays can hand them over
unchanged.  These dtypes are byte-compatible with (sizes/offsets checked
against the reference build in tests/test_layout.py):

* ``Float3``                Quantom/Quantom/QuantomTypes.cuh:33-168   (12 B)
* ``Solvent``               Quantom/Quantom/Bodies.cuh:19-25          (24 B)
* ``PairBond``              Bodies.cuh:61-85                          (16 B)
* ``AngleBond``             Bodies.cuh:87-98                          (20 B)
* ``DihedralBond``          Bodies.cuh:100-113                        (28 B)
* ``LJ_Ignores``            Bodies.cuh:169-198                        (65 B)
* ``CompoundState``         Bodies.cuh:303-315                        (772 B)
* ``Compound``              Bodies.cuh:318-472 (LIMA_DEBUGMODE on)    (24,036 B)
* ``ParticleRefCompact``    Bodies.cuh:644-650                        (8 B)
* ``CompoundBridgeCompact`` Bodies.cuh:652-725                        (2,352 B)
* ``ParticleParameters``    Forcefield.cuh:18-22; ``ForceField`` :25-27 (384 B)

Units are the reference's: nm, ns, kg/mol, J/mol.
"""
import numpy as np

MAX_COMPOUND_PARTICLES = 64          # Constants.cuh:58
MAX_PAIRBONDS = 128                  # Bodies.cuh:300
MAX_ANGLEBONDS = 256                 # Bodies.cuh:301
MAX_DIHEDRALS = 384                  # Bodies.cuh:302
LJ_IGNORES_MAX = 32                  # Bodies.cuh:170
MAX_PARTICLES_IN_BRIDGE = 32         # Constants.cuh:110
MAX_SINGLEBONDS_IN_BRIDGE = 32       # Constants.cuh:111
MAX_ANGLEBONDS_IN_BRIDGE = 32        # Constants.cuh:112
MAX_DIHEDRALBONDS_IN_BRIDGE = 32     # Constants.cuh:113
MAX_ATOM_TYPES = 32                  # Forcefield.cuh:12
MAX_COMPOUNDS = 0xFF                 # Constants.cuh:88 (LJ_Ignores stores uint8 compound ids)
ATOMTYPE_SOL = 0                     # Forcefield.cuh:15

float3 = np.dtype((np.float32, 3))

Solvent = np.dtype([("pos", float3), ("pos_tsub1", float3)])

PairBond = np.dtype({"names": ["b0", "kb", "atom_indexes"],
                     "formats": [np.float32, np.float32, (np.uint32, 2)],
                     "offsets": [0, 4, 8], "itemsize": 16})

AngleBond = np.dtype({"names": ["theta_0", "k_theta", "atom_indexes"],
                      "formats": [np.float32, np.float32, (np.uint32, 3)],
                      "offsets": [0, 4, 8], "itemsize": 20})

DihedralBond = np.dtype({"names": ["phi_0", "k_phi", "n", "atom_indexes"],
                         "formats": [np.float32, np.float32, np.uint8, (np.uint32, 4)],
                         "offsets": [0, 4, 8, 12], "itemsize": 28})

LJ_Ignores = np.dtype({"names": ["local_ids", "compound_ids", "n_ignores"],
                       "formats": [(np.uint8, LJ_IGNORES_MAX), (np.uint8, LJ_IGNORES_MAX), np.uint8],
                       "offsets": [0, 32, 64], "itemsize": 65})

CompoundState = np.dtype({"names": ["positions", "n_particles"],
                          "formats": [(float3, MAX_COMPOUND_PARTICLES), np.uint8],
                          "offsets": [0, 768], "itemsize": 772})

Compound = np.dtype({
    "names": ["n_particles", "prev_positions", "forces", "atom_types", "atom_color_types",
              "lj_ignore_list", "particle_global_ids", "center_of_mass",
              "n_singlebonds", "singlebonds", "n_anglebonds", "anglebonds",
              "n_dihedrals", "dihedrals", "key_particle_index", "confining_particle_sphere"],
    "formats": [np.uint8, (float3, 64), (float3, 64), (np.uint8, 64), (np.uint8, 64),
                (LJ_Ignores, 64), (np.uint32, 64), float3,
                np.uint16, (PairBond, MAX_PAIRBONDS), np.uint16, (AngleBond, MAX_ANGLEBONDS),
                np.uint16, (DihedralBond, MAX_DIHEDRALS), np.int32, np.float32],
    "offsets": [0, 4, 772, 1540, 1604, 1668, 5828, 6084,
                6096, 6100, 8148, 8152, 13272, 13276, 24028, 24032],
    "itemsize": 24036})

ParticleRefCompact = np.dtype([("compound_id", np.int32), ("local_id_compound", np.int32)])

CompoundBridgeCompact = np.dtype({
    "names": ["particle_refs", "atom_types", "n_particles", "n_singlebonds", "singlebonds",
              "n_anglebonds", "anglebonds", "n_dihedrals", "dihedrals"],
    "formats": [(ParticleRefCompact, 32), (np.uint8, 32), np.int32, np.uint16,
                (PairBond, MAX_SINGLEBONDS_IN_BRIDGE), np.uint16, (AngleBond, MAX_ANGLEBONDS_IN_BRIDGE),
                np.uint16, (DihedralBond, MAX_DIHEDRALBONDS_IN_BRIDGE)],
    "offsets": [0, 256, 288, 292, 296, 808, 812, 1452, 1456],
    "itemsize": 2352})

ParticleParameters = np.dtype([("mass", np.float32), ("sigma", np.float32), ("epsilon", np.float32)])
# RenderBall (QuantomTypes.cuh:362-369) = lima_render_ball, 32 bytes
RenderBall = np.dtype([("pos", float3), ("radius", np.float32), ("color", np.int32, 3), ("disable", np.uint8),
                       ("pad", np.uint8, 3)])
# atom_color_types index -> ATOM_TYPE (Rasterizer.cu:126-146; QuantomTypes.cuh:16
# NONE 0, O 1, C 2, P 3, N 4, H 5, SOL 6)
RENDER_TYPE_OF_COLOR = (6, 2, 1, 4, 5, 3, 6)
ForceField = np.dtype([("particle_parameters", (ParticleParameters, MAX_ATOM_TYPES))])

# Offsets the tests compare with the reference build (ref_layout ids).
REF_LAYOUT_IDS = {
    0: ("Float3", 12), 1: ("Solvent", Solvent.itemsize), 2: ("CompoundState", CompoundState.itemsize),
    3: ("Compound", Compound.itemsize), 5: ("LJ_Ignores", LJ_Ignores.itemsize),
    6: ("PairBond", PairBond.itemsize), 7: ("AngleBond", AngleBond.itemsize),
    8: ("DihedralBond", DihedralBond.itemsize), 9: ("CompoundBridgeCompact", CompoundBridgeCompact.itemsize),
    10: ("ForceField", ForceField.itemsize), 11: ("ParticleRefCompact", ParticleRefCompact.itemsize),
}
REF_OFFSET_IDS = {
    20: (Compound, "prev_positions"), 21: (Compound, "forces"), 22: (Compound, "atom_types"),
    23: (Compound, "atom_color_types"), 24: (Compound, "lj_ignore_list"),
    25: (Compound, "particle_global_ids"), 26: (Compound, "center_of_mass"),
    27: (Compound, "n_singlebonds"), 28: (Compound, "singlebonds"), 29: (Compound, "n_anglebonds"),
    30: (Compound, "anglebonds"), 31: (Compound, "n_dihedrals"), 32: (Compound, "dihedrals"),
    33: (Compound, "key_particle_index"), 34: (Compound, "confining_particle_sphere"),
    40: (CompoundBridgeCompact, "particle_refs"), 41: (CompoundBridgeCompact, "atom_types"),
    42: (CompoundBridgeCompact, "n_particles"), 43: (CompoundBridgeCompact, "n_singlebonds"),
    44: (CompoundBridgeCompact, "singlebonds"), 45: (CompoundBridgeCompact, "n_anglebonds"),
    46: (CompoundBridgeCompact, "anglebonds"), 47: (CompoundBridgeCompact, "n_dihedrals"),
    48: (CompoundBridgeCompact, "dihedrals"), 50: (DihedralBond, "n"), 51: (DihedralBond, "atom_indexes"),
}
