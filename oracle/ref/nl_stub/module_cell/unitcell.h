// Test infrastructure (oracle): stand-in for the reference's UnitCell (module_cell/unitcell.h) when its
// Nonlocal operator (module_hamilt_pw/hamilt_pwdft/operator_pw/nonlocal_pw.cpp) is compiled from its source.
// That operator reads three things of the cell: the number of atom types, the atoms of each type and the
// beta functions of each atom's pseudopotential (ucell->ntype, atoms[it].na, atoms[it].ncpp.nh), so this
// header declares exactly those; the real class pulls in the whole cell, symmetry and I/O layers.
#ifndef UNITCELL_H
#define UNITCELL_H

struct OracleNcpp {
    int nh = 0;  // beta functions (projectors) per atom of the type
};

class Atom {
  public:
    int na = 0;  // atoms of the type
    OracleNcpp ncpp;
};

class UnitCell {
  public:
    int ntype = 0;
    Atom* atoms = nullptr;
};

#endif
