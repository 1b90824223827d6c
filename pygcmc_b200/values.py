"""Packed numpy dtypes of the GCMC state arrays and the reference's physical constants.

The dtypes are byte-identical to the C structs that cross the native boundary
(pyGCMC ``gcmc/python/values.py:18-62`` mirrors ``gcmc/cpp/gcmc.h:47-100``):

=================  =======  ==========================================
dtype              bytes    C struct
=================  =======  ==========================================
``Atom_dtype``     20       ``Atom {float position[3]; float charge; int type;}``
``AtomArray_dtype`` 436     ``AtomArray`` (fragment type, <= 20 sites)
``Info_dtype``     76       ``InfoStruct``
``Residue_dtype``  20       ``residue {float position[3]; int atomNum; int atomStart;}``
=================  =======  ==========================================
"""
import numpy as np

# gcmc/cpp/gcmc.h:28-41
TEMPERATURE = 300.0
BOLTZMANN = 0.0083115  # kJ/mol/K
BETA = 1.0 / (BOLTZMANN * TEMPERATURE)
MOLES_TO_MOLECULES = 0.0006023  # mol/L -> molecules/A^3
KCAL_TO_KJ = 4.184
COULOMB = 1388.431112  # kJ/mol * A / e^2, gcmc/cpp/gcmc_energy.h:137
MAX_SITES = 20  # AtomArray.atoms[20]

Atom_dtype = np.dtype([
    ("position", np.float32, (3,)),
    ("charge", np.float32),
    ("type", np.int32),
])

AtomArray_dtype = np.dtype([
    ("name", "S4"),
    ("startRes", np.int32),
    ("muex", np.float32),
    ("conc", np.float32),
    ("confBias", np.int32),
    ("mcTime", np.float32),
    ("totalNum", np.int32),
    ("maxNum", np.int32),
    ("num_atoms", np.int32),
    ("atoms", Atom_dtype, (MAX_SITES,)),
])

Info_dtype = np.dtype([
    ("mcsteps", np.int32),
    ("cutoff", np.float32),
    ("grid_dx", np.float32),
    ("startxyz", np.float32, (3,)),
    ("cryst", np.float32, (3,)),
    ("showInfo", np.int32),
    ("cavityFactor", np.float32),
    ("fragTypeNum", np.int32),
    ("totalGridNum", np.int32),
    ("totalResNum", np.int32),
    ("totalAtomNum", np.int32),
    ("ffXNum", np.int32),
    ("ffYNum", np.int32),
    ("PME", np.int32),
    ("seed", np.uint32),
])

Residue_dtype = np.dtype([
    ("position", np.float32, (3,)),
    ("atomNum", np.int32),
    ("atomStart", np.int32),
])

# Per-step record written by the engine (and by the CPU oracle), 48 bytes.
StepLog_dtype = np.dtype([
    ("step", np.int32), ("move", np.int32), ("ftype", np.int32), ("k", np.int32),
    ("n_before", np.int32), ("n_after", np.int32), ("n_clusters", np.int32), ("n_accept", np.int32),
    ("first_accept", np.int32), ("slot", np.int32), ("e_sum", np.float64), ("e_total", np.float64),
])

assert Atom_dtype.itemsize == 20
assert AtomArray_dtype.itemsize == 436
assert Info_dtype.itemsize == 76
assert Residue_dtype.itemsize == 20
assert StepLog_dtype.itemsize == 56
