#pragma once

namespace maple {

extern const int kCorner[8][3];

// FP64 element tables for a voxel of edge 1 (r = 1).
struct ElementTables {
  double Ke3[24 * 24];  // elastic element stiffness
  double Fe3[24 * 6];   // elastic element load for the 6 unit macro strains
  double X03[24 * 6];   // elastic element reference field (Ke3 X03 = Fe3, pinned)
  double KX3[24 * 6];   // Ke3 X03
  double Ke1[8 * 8];    // conduction element stiffness
  double Fe1[8 * 3];
  double X01[8 * 3];
  double KX1[8 * 3];
  double W[8 * 8 * 8];      // child prolongation weights W[c][a][b]
  double M3[8 * 24 * 24];   // W_c^T Ke3 W_c
  double M1[8 * 8 * 8];     // W_c^T Ke1 W_c
  double lam_elem[2];       // lambda_max(D_e^-1 K_e): [elastic, thermal]
};

void element_tables(double E, double nu, double kappa, ElementTables* t);

}  // namespace maple
