// Internal declarations shared by the host setup code and the CUDA kernels of
// libfem25gpu.  Not part of the public ABI (include/fem25gpu.h is).
#pragma once
#include <cstdint>
#include <string>
#include <vector>

#include "fem25gpu.h"

namespace fem25 {

constexpr int kNord = 4;                 // NORD: degree-4 GLL elements
constexpr int kNl = kNord + 1;           // NLXI = NLETA = 5
constexpr int kNen = kNl * kNl;          // 25 element nodes
constexpr int kNee = 3 * kNen;           // 75 element equations
constexpr int kNint = 2 * kNord + 2 + 3; // 13 Lobatto points (asmble.f90:110-112)
constexpr int kNq = kNint * kNint;       // 169 quadrature points
constexpr int kNab = kNen * kNen;        // 625 node pairs per element

// Quadrature tables built on the host once (DSHL, dshl.f:1-243).
struct Tables {
  double xigll[kNint];   // XIGLL(:,1), midpoint forced to 0
  double wts[kNint];     // XIGLL(:,2)
  double xipts[kNl];     // GLL interpolation points, midpoint 0
  // SHL(3,NEN,NINT,NINT) column-major: shl[((intz*kNint+intx)*kNen + a)*3 + k]
  double shl[3 * kNen * kNq];
  // bilinear anchor shape functions at the quadrature points (CSF2D)
  double sf[kNq][4];
  double dsf[kNq][2][4];
};
void build_tables(Tables *t);
void lobatto(int n, double *x, double *w);

// Host graph (GEN_GRAPH25 products).
struct HostGraph {
  int nelem = 0, nnp = 0, ndof = 0;
  long long nzero = 0;
  std::vector<int> ien;    // IEN(NEN,NELEM)
  std::vector<int> lm;     // LM(3,NEN,NELEM)
  std::vector<int> irptr;  // IRPTR(NDOF+1)
  std::vector<int> jcptr;  // JCPTR(NZERO)
  std::vector<char> cnp;   // CNP(NDOF)
};
int build_graph(const fem25_mesh *m, HostGraph *g, std::string *err);

// 3x3 block view of the CSR: every node holds three consecutive DOFs (GENID
// numbers the components of a node together and fixes all three at once),
// so row 3A+i has the same node columns for i = 0,1,2.
struct BlockCSR {
  int nbrow = 0;               // DOF nodes = NDOF/3
  long long nblocks = 0;
  std::vector<long long> brptr;   // [nbrow+1]
  std::vector<int> bcol;          // [nblocks] block column (0-based node)
  std::vector<int> brow;          // [nblocks] block row
};
int build_block_csr(int ndof, long long nzero, const int *irptr, const int *jcptr, BlockCSR *b,
                    std::string *err);

// Reference-compatible gradient set-up (GENGMASK, ELEM_WTS, GRADPTRS).
struct RefGradSetup {
  int ncon = 0, nnpinv = 0;
  long long nz = 0;
  std::vector<int> maskg;    // MASKG(NNPG)
  std::vector<int> mconn;    // MCONN(NNPG,NCON) column-major
  std::vector<double> elem_wts;
  std::vector<int> jcsc, icsc;
  std::vector<int> anchor_of_col;  // 0-based anchor of each CSC column
};
int build_ref_grad(const fem25_mesh *m, const int *lm, RefGradSetup *r, std::string *err);

}  // namespace fem25
