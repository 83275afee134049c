// C entry points over the reference's own matrix.cpp (dense LU inverse),
// elastic.cpp (ElasticMaterial: readModuli fills the compliance, the
// stiffness is its inverse), pStress.cpp (PlaneStress) and
// heatTransferMaterial.cpp (readConductivity, the flux) and node.cpp
// (setNumDofPerNode, the node records), compiled
// unmodified into oracle/_ref/libbeta_ref_material.so.  Test infrastructure:
// used only to pin the oracle's constitutive matrices against the
// reference's code.  The materials read their constants from an input
// stream, so each entry point writes the constants the way an input deck
// holds them and lets the reference's read() parse them.
#include <cstdio>
#include <cstring>
#include <sstream>
#include <strings.h>

#include "elastic.hpp"
#include "heatTransferMaterial.hpp"
#include "node.hpp"
#include "pStress.hpp"

int verboseFlag = 0;

// The input helpers elastic.cpp calls (utility.cpp is not compiled here):
// read the next non-blank line that is not a // comment, split it at blanks
// into tokenList, and return 1 when its first token is terminateString (or
// the input ends), 0 otherwise.
int getLineAndTokenize(std::istream* in, char* terminateString, char* tokenList[], int& numberOfTokens) {
  static char line[1024];
  for (;;) {
    numberOfTokens = 0;
    if (!in->getline(line, sizeof line)) return 1;
    char* save = nullptr;
    for (char* t = strtok_r(line, " \t\r", &save); t && numberOfTokens < 20; t = strtok_r(nullptr, " \t\r", &save))
      tokenList[numberOfTokens++] = t;
    if (numberOfTokens == 0 || std::strncmp(tokenList[0], "//", 2) == 0) continue;
    return strcasecmp(tokenList[0], terminateString) == 0 ? 1 : 0;
  }
}
void banner(char*, std::ostream&) {}

namespace {
// The materials print what they read; keep that out of the caller's stdout.
struct QuietCout {
  std::stringstream sink;
  std::streambuf* old;
  QuietCout() : old(std::cout.rdbuf(sink.rdbuf())) {}
  ~QuietCout() { std::cout.rdbuf(old); }
};

// ElasticMaterial::initialize + read of a "readModuli" block holding m9.
bool read_ortho(ElasticMaterial& m, const double* m9) {
  m.initialize();
  std::ostringstream deck;
  char num[40];
  deck << "readModuli\n";
  for (int i = 0; i < 9; ++i) {
    std::snprintf(num, sizeof num, "%.17g ", m9[i]);
    deck << num;
  }
  deck << "\nexitElasticMaterial\n";
  std::istringstream in(deck.str());
  return m.read(&in);
}
}  // namespace

extern "C" {
// Matrix::invert (ludcmp + lubksb) of an n x n row-major matrix, in place.
int ref_matrix_invert(int n, double* A) {
  Matrix M(n, n);
  for (int i = 0; i < n; ++i)
    for (int j = 0; j < n; ++j) M(i, j) = A[i * n + j];
  M.invert();
  for (int i = 0; i < n; ++i)
    for (int j = 0; j < n; ++j) A[i * n + j] = M(i, j);
  return 0;
}

// ElasticMaterial::initialize + read of a "readModuli" block with the nine
// constants m9 = (E11, E22, E33, nu12, nu23, nu13, G12, G23, G13); C36 gets
// the material's stiffness (cMat, row-major 6 x 6) and S36, when non-null,
// its compliance.
int ref_cmat_ortho3d(const double* m9, double* C36, double* S36) {
  QuietCout q;
  ElasticMaterial m;
  if (!read_ortho(m, m9)) return 1;
  for (int i = 0; i < 6; ++i)
    for (int j = 0; j < 6; ++j) {
      C36[i * 6 + j] = (*m.cMat)(i, j);
      if (S36) S36[i * 6 + j] = (*m.S)(i, j);
    }
  return 0;
}

// PlaneStress::initialize + read of (E11, E22, nu12, G12) (the two thermal
// coefficients zero); C9 gets its stiffness (row-major 3 x 3).
int ref_cmat_plane_stress(const double* m4, double* C9) {
  QuietCout q;
  PlaneStress p;
  p.initialize();
  char deck[256];
  std::snprintf(deck, sizeof deck, "%.17g %.17g %.17g %.17g 0 0\n", m4[0], m4[1], m4[2], m4[3]);
  std::istringstream in(deck);
  if (!p.read(&in)) return 1;
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) C9[i * 3 + j] = (*p.cMat)(i, j);
  return 0;
}

// HeatTransferMaterial::initialize + read of a readConductivity block
// (k11, k22, k33): C9 gets its conductivity tensor (row-major 3 x 3) and,
// for the temperature gradient grad, flux = calculateFlux (-k grad T).
int ref_heat_conductivity(const double* k3, const double* grad, double* C9, double* flux) {
  QuietCout q;
  HeatTransferMaterial mat;
  mat.initialize();
  char deck[256];
  std::snprintf(deck, sizeof deck, "readConductivity\n%.17g %.17g %.17g\nexitHeatTransferMaterial\n", k3[0],
                k3[1], k3[2]);
  std::istringstream in(deck);
  if (!mat.read(&in)) return 1;
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) C9[i * 3 + j] = (*mat.cMat)(i, j);
  InterpAndSolDerivatives id;
  id.p_u1_x1 = grad[0];
  id.p_u1_x2 = grad[1];
  id.p_u1_x3 = grad[2];
  mat.calculateFlux(flux, &id);
  return 0;
}

// Node::setNumDofPerNode over numNodes nodes reading the block deck (lines
// "n all" or "n first last increment", ended by "end"): numDof and firstDof
// per node and the total.  Returns 0.
int ref_set_num_dof(int numNodes, const char* deck, int* numDof, int* firstDof, int* total) {
  QuietCout q;
  NodeGroup nodes(numNodes);
  for (int i = 0; i < numNodes; ++i) nodes[i].nodeNum = i;
  std::istringstream in(deck);
  std::ostringstream out;
  int tot = 0;
  Node::setNumDofPerNode(&in, &out, numNodes, &nodes, tot);
  for (int i = 0; i < numNodes; ++i) {
    numDof[i] = nodes[i].getNumDof();
    firstDof[i] = nodes[i].getFirstDof();
  }
  *total = tot;
  return 0;
}

// Node::writeBinary of nodes (numbers nums, coordinates xyz n x 3) to path,
// one record after another, and Node::readBinary of them back into
// nums_back / xyz_back.
int ref_node_records(int n, const int* nums, const double* xyz, const char* path, int* nums_back,
                     double* xyz_back) {
  FILE* f = std::fopen(path, "wb");
  if (!f) return 1;
  for (int i = 0; i < n; ++i) {
    Node nd(nums[i], xyz[3 * i], xyz[3 * i + 1], xyz[3 * i + 2]);
    nd.writeBinary(f);
  }
  std::fclose(f);
  f = std::fopen(path, "rb");
  if (!f) return 1;
  for (int i = 0; i < n; ++i) {
    Node nd;
    nd.readBinary(f);
    nums_back[i] = nd.nodeNum;
    xyz_back[3 * i] = nd.x;
    xyz_back[3 * i + 1] = nd.y;
    xyz_back[3 * i + 2] = nd.z;
  }
  std::fclose(f);
  return 0;
}

// ElasticMaterial::calculateStress at zero temperature and moisture: the
// stress of a strain (6, engineering shear) for the material of m9.
int ref_elastic_stress(const double* m9, const double* strain, double* stress) {
  QuietCout q;
  ElasticMaterial m;
  if (!read_ortho(m, m9)) return 1;
  ElasticISV isv;
  Rotation identity;
  double eps[6];
  for (int i = 0; i < 6; ++i) eps[i] = strain[i];
  m.calculateStress(stress, eps, &isv, &identity);
  return 0;
}
}
