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
  // level-2 element matrix of one fine element of unit density at position
  // f = (4 fx + fy) 4 + fz of the level-2 element's 4^3 fine elements:
  // G_f = (W_c1 (x) I)^T M_c0 (W_c1 (x) I), c1 = the level-1 child (f / 2 per
  // axis), c0 = the fine element inside it (f % 2 per axis)
  double G3[64 * 24 * 24];
  double G1[64 * 8 * 8];
  double lam_elem[2];       // lambda_max(D_e^-1 K_e): [elastic, thermal]
};

void element_tables(double E, double nu, double kappa, ElementTables* t);

}  // namespace maple
