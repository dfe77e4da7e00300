// Fusion pattern per expression instance in the per-Gaussian and per-pixel
// arithmetic (see s1/s2/d2/s3 in common.cuh).  Established by comparing
// against the reference extension's buffers on a B200: with these values
// depth, screen position, 3-D covariance, conic, colour, radius and tile
// counts are bit-identical to the reference, and so are contributor counts,
// alpha and depth images when blending the same sorted lists.  Indices:
// RQ = rotation matrix entries (column-major), SIGMA = stored covariance
// entries, VIEW/PROJ rows, DPROJ = Jacobian rows (x then y), SIGV = Sigma*j
// rows, DOT3 = cxx/cxy/cyy, PIX = screen x/y, BL_* = per-pixel Gaussian
// evaluation, SH* = colour polynomial terms.  The CPU oracle carries the
// same table.
#pragma once

namespace w2w {
namespace fp {
constexpr int RQ0 = 0;
constexpr int RQ1 = 1;
constexpr int RQ2 = 2;
constexpr int RQ3 = 1;
constexpr int RQ4 = 1;
constexpr int RQ5 = 1;
constexpr int RQ6 = 2;
constexpr int RQ7 = 1;
constexpr int RQ8 = 1;
constexpr int SIGMA0 = 1;
constexpr int SIGMA1 = 1;
constexpr int SIGMA2 = 1;
constexpr int SIGMA3 = 1;
constexpr int SIGMA4 = 1;
constexpr int SIGMA5 = 1;
constexpr int VIEW_A0 = 1;
constexpr int VIEW_A1 = 1;
constexpr int VIEW_A2 = 1;
constexpr int VIEW_A3 = 1;
constexpr int VIEW_B0 = 1;
constexpr int VIEW_B1 = 1;
constexpr int VIEW_B2 = 1;
constexpr int VIEW_B3 = 1;
constexpr int RAYR2 = 1;
constexpr int DPROJ0 = 1;
constexpr int DPROJ1 = 1;
constexpr int DPROJ2 = 1;
constexpr int DPROJ3 = 1;
constexpr int DPROJ4 = 1;
constexpr int DPROJ5 = 1;
constexpr int SIGV0 = 1;
constexpr int SIGV1 = 1;
constexpr int SIGV2 = 1;
constexpr int SIGV3 = 1;
constexpr int SIGV4 = 1;
constexpr int SIGV5 = 1;
constexpr int DOT30 = 1;
constexpr int DOT31 = 1;
constexpr int DOT32 = 1;
constexpr int DET = 1;
constexpr int PROJ_A0 = 1;
constexpr int PROJ_A1 = 1;
constexpr int PROJ_A2 = 1;
constexpr int PROJ_A3 = 1;
constexpr int PROJ_B0 = 1;
constexpr int PROJ_B1 = 1;
constexpr int PROJ_B2 = 1;
constexpr int PROJ_B3 = 1;
constexpr int PIX0 = 2;
constexpr int PIX1 = 2;
constexpr int ADR_DELTA = 1;
constexpr int BL_DET = 1;
constexpr int BL_TX = 1;
constexpr int BL_TY = 2;
constexpr int BL_NUM = 2;
constexpr int BL_DEPTH = 1;
constexpr int SH_DOT = 1;
constexpr int SH_ACC = 1;
constexpr int SH2A = 0;
constexpr int SH2B = 0;
constexpr int SH3A = 1;
constexpr int SH3B = 0;
constexpr int SH3C = 1;
constexpr int SH3D = 0;
constexpr int SH3E = 1;
}  // namespace fp
}  // namespace w2w
