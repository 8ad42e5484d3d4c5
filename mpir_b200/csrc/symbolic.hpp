// Host symbolic analysis for the LDL^T factorization of a quasidefinite
// matrix given by its upper triangle in CSC.
//
//  * fill-reducing permutation (absent from the reference, which factors in
//    natural order): positive-diagonal unknowns first, ordered by recursive
//    level-set nested dissection of their graph, then the remaining unknowns;
//    the result is post-ordered on its elimination tree;
//  * elimination tree and per-column counts of L, equal element for element
//    to QDLDL_etree on the permuted matrix (qdldl.hpp:48-105);
//  * supernodes (maximal column runs with nested structure) and their row
//    structures, which give the L pattern of QDLDL_factor (qdldl.hpp:172-345)
//    column by column;
//  * the multifrontal schedule the GPU numeric factor and solves run:
//    etree levels, children lists, relative row maps, the scatter map of A's
//    entries into the factor panels and an arena plan for the update
//    matrices.
#pragma once
#include <cstdint>
#include <string>
#include <vector>

namespace mpir {

// Fronts with at most this many rows are factored whole in shared memory,
// one thread block per front; larger fronts go through the blocked path.
constexpr int kSmallFront = 64;
// Column-block width of the blocked dense partial factorization.
constexpr int kNB = 128;

struct Symbolic {
  int64_t n   = 0;
  int64_t nnz = 0;  // entries of the caller's upper triangle

  // perm[new] = old, iperm[old] = new.
  std::vector<int64_t> perm, iperm;

  // Permuted upper CSC (sorted rows) and, per entry, its index in the
  // caller's Ax: the exact input QDLDL_factor would get for P K P^T.
  std::vector<int64_t> Cp, Ci, Csrc;

  // Elimination tree (-1 for roots) and below-diagonal counts of L.
  std::vector<int64_t> etree, Lnz;
  int64_t              nnzL = 0;

  // Supernodes: columns [sfirst[J], sfirst[J+1]).  Row index set of J is
  // srows[srowptr[J] .. srowptr[J+1]) = its own columns then R_J ascending.
  int64_t              ns = 0;
  std::vector<int64_t> sfirst, sparent, srowptr, col2sup;
  std::vector<int32_t> srows;
  // Panel of J: h x w column-major floats at slofs[J] (h rows, w columns).
  std::vector<int64_t> slofs;
  int64_t              panel_elems = 0;
  // For each J with a parent: local row in the parent's index set of each of
  // J's R_J rows, at srel[srowptr[J] + w_J + a].
  std::vector<int32_t> srel;

  // Levels: level 0 = supernodes without children.  Supernodes grouped by
  // level in level_sup[level_ptr[t] .. level_ptr[t+1]).
  int32_t              nlevels = 0;
  std::vector<int32_t> slevel;
  std::vector<int64_t> level_ptr;
  std::vector<int32_t> level_sup;
  // Children of J: child_list[child_ptr[J] .. child_ptr[J+1]).
  std::vector<int64_t> child_ptr;
  std::vector<int32_t> child_list;

  // Update matrix U_J (|R_J| x |R_J|, column-major) at uofs[J] floats in the
  // update arena; -1 when R_J is empty.  Arena size in floats.
  std::vector<int64_t> uofs;
  int64_t              uarena_elems = 0;

  // Per-entry scatter target of the caller's entry p in the panel storage.
  std::vector<int64_t> amap;
  // Caller's row / column of entry p and position of each caller column's
  // diagonal entry (-1 if absent): used for the symmetric scaling.
  std::vector<int32_t> arow, acol;
  std::vector<int64_t> diag_pos;

  // Full symmetric CSR of P K P^T (both triangles), each entry's index in the
  // caller's Ax.
  std::vector<int64_t> Kp, Ksrc;
  std::vector<int32_t> Kj;

  // Solve workspace: front vector of J at zofs[J] (h_J doubles).
  std::vector<int64_t> zofs;
  int64_t              z_elems = 0;

  // Largest front height and width.
  int64_t max_h = 0, max_w = 0;

  int64_t w(int64_t J) const { return sfirst[J + 1] - sfirst[J]; }
  int64_t h(int64_t J) const { return srowptr[J + 1] - srowptr[J]; }
};

// Status codes shared with the C ABI (0 = success).
enum : int {
  kOk          = 0,
  kBadInput    = -1,  // not upper triangular, empty column, zero pivot
  kOverflow    = -2,  // nnz(L) overflows
  kBadArgument = -6,
};

// Ordering choice.
enum class Ordering : int { Natural = 0, Auto = 1 };

// Analyse an upper-CSC matrix.  diag_sign (optional, length n, caller order)
// marks unknowns whose diagonal is positive (1) or not (0); with
// Ordering::Auto these split the ordering into the two blocks.  Returns a
// status code; on error `err` holds a message.
int analyze(int64_t n, const int64_t *Ap, const int64_t *Ai,
            const int8_t *diag_sign, Ordering ord, Symbolic &S,
            std::string &err);

// Build the supernodal schedule from a factor pattern given as QDLDL's CSC
// L (natural order, no permutation).  Used by the QDLDL_solve entry point.
int analyze_from_L(int64_t n, const int64_t *Lp, const int64_t *Li,
                   Symbolic &S, std::string &err);

// Elimination tree and column counts of an upper-CSC matrix (no ordering).
// Returns sum(Lnz) or a negative status like QDLDL_etree.
int64_t etree_counts(int64_t n, const int64_t *Ap, const int64_t *Ai,
                     int64_t *etree, int64_t *Lnz);

}  // namespace mpir
