// Host sparsity-pattern build for general dof tables (any mesh, any dof numbering).
//
// Produces the arrays of the reference's patternbuild.build_tables
// (hippymfem/fem/patternbuild.py:209-253): CSR rows holding each distinct column once,
// the diagonal first on a square pattern (hypre's order) and the other columns
// ascending, and for every element entry k = (e*ndt + a)*ndr + b its position in the
// values array.
//
// How it is done here:
//   1. incidence: the (element, local row) items of each global row, by a stable
//      counting sort of the test table (items of a row in ascending (e, a));
//   2. per row, independently (rows are split over host threads): the columns of all
//      the row's items are copied into a small buffer, sorted and made unique -- that
//      is the row's column set, ascending; with diag_first the diagonal, if present,
//      is rotated to the front;
//   3. each entry's position is found by a binary search of its column in the
//      ascending set, shifted by one for the columns that precede the diagonal.
// The per-row work is bounded by (items of the row) x ndr, so no array of the column
// range is needed and memory stays proportional to the table.
#include <algorithm>
#include <cstdint>
#include <thread>
#include <vector>

#include "../../include/hippymfem_b200.h"

namespace {

// rows -> their (e*ndt + a) items, ascending; start has nrow + 1 entries
struct RowItems {
  std::vector<int64_t> start;
  std::vector<int64_t> item;
};

int row_items(const int64_t* tdofs, int64_t nitem, int64_t nrow, RowItems& ri) {
  std::vector<int64_t> next(nrow + 1, 0);
  for (int64_t i = 0; i < nitem; ++i) {
    const int64_t r = tdofs[i];
    if (r < 0 || r >= nrow) return HM_ERR_RANGE;
    ++next[r + 1];
  }
  for (int64_t r = 0; r < nrow; ++r) next[r + 1] += next[r];
  ri.start = next;                       // row r's items are [start[r], start[r + 1])
  ri.item.resize(nitem);
  for (int64_t i = 0; i < nitem; ++i) ri.item[next[tdofs[i]]++] = i;
  return HM_OK;
}

// The rows [r0, r1): count[r] = distinct columns; with indices/slot given (and indptr
// holding the final row offsets) also the columns and every entry's position.
// Returns false on a column outside [0, ncol).
bool build_rows(const int64_t* cdofs, int ndt, int ndr, int64_t ncol, bool diag_first,
                const RowItems& ri, int64_t r0, int64_t r1, int64_t* count,
                const int32_t* indptr, int32_t* indices, int32_t* slot) {
  std::vector<int64_t> cols;
  for (int64_t r = r0; r < r1; ++r) {
    cols.clear();
    for (int64_t p = ri.start[r]; p < ri.start[r + 1]; ++p) {
      const int64_t* crow = cdofs + (ri.item[p] / ndt) * ndr;
      for (int b = 0; b < ndr; ++b) {
        if (crow[b] < 0 || crow[b] >= ncol) return false;
        cols.push_back(crow[b]);
      }
    }
    std::sort(cols.begin(), cols.end());
    cols.erase(std::unique(cols.begin(), cols.end()), cols.end());
    const int64_t nc = (int64_t)cols.size();
    count[r] = nc;
    if (indices == nullptr) continue;
    // the diagonal's place in the ascending set (-1: absent or not wanted first)
    int64_t kd = -1;
    if (diag_first) {
      auto it = std::lower_bound(cols.begin(), cols.end(), r);
      if (it != cols.end() && *it == r) kd = it - cols.begin();
    }
    // ascending order with the diagonal moved ahead: column k of the ascending set sits
    // at k + 1 if it precedes the diagonal, at 0 if it is the diagonal, at k after it
    auto place = [&](int64_t k) { return k == kd ? 0 : (k < kd ? k + 1 : k); };
    const int64_t base = indptr[r];
    for (int64_t k = 0; k < nc; ++k) indices[base + place(k)] = (int32_t)cols[k];
    for (int64_t p = ri.start[r]; p < ri.start[r + 1]; ++p) {
      const int64_t it = ri.item[p];
      const int64_t* crow = cdofs + (it / ndt) * ndr;
      int32_t* sl = slot + it * ndr;
      for (int b = 0; b < ndr; ++b) {
        const int64_t k = std::lower_bound(cols.begin(), cols.end(), crow[b]) - cols.begin();
        sl[b] = (int32_t)(base + place(k));
      }
    }
  }
  return true;
}

// f(r0, r1) over contiguous row ranges on up to nthreads host threads; false if any
// range returned false
template <typename F>
bool over_rows(int64_t nrow, int nthreads, F&& f) {
  int nt = nthreads > 0 ? nthreads : (int)std::max(1u, std::thread::hardware_concurrency());
  if (nrow < 8192) nt = 1;
  const int64_t chunk = (nrow + nt - 1) / std::max(nt, 1);
  std::vector<char> ok(nt, 1);
  std::vector<std::thread> pool;
  for (int i = 0; i < nt; ++i) {
    const int64_t a = i * chunk, b = std::min(nrow, a + chunk);
    if (a >= b) break;
    pool.emplace_back([&, i, a, b] { ok[i] = f(a, b) ? 1 : 0; });
  }
  for (auto& t : pool) t.join();
  return std::all_of(ok.begin(), ok.end(), [](char c) { return c != 0; });
}

}  // namespace

extern "C" int hm_pattern_build(const int64_t* tdofs, const int64_t* cdofs, int64_t ne, int ndt,
                                int ndr, int64_t nrow, int64_t ncol, int diag_first, int nthreads,
                                int32_t* indptr, int32_t* indices, int64_t indices_capacity,
                                int32_t* slot, int64_t* nnz) {
  if (ne < 0 || ndt <= 0 || ndr <= 0 || nrow < 0 || ncol < 0 || !indptr || !nnz) return HM_ERR_ARG;
  if ((ne > 0 && (!tdofs || !cdofs)) || ((indices == nullptr) != (slot == nullptr))) return HM_ERR_ARG;
  if (ne * (int64_t)ndt * ndr > INT32_MAX) return HM_ERR_UNSUPPORTED;
  RowItems ri;
  const int rc = row_items(tdofs, ne * (int64_t)ndt, nrow, ri);
  if (rc) return rc;
  std::vector<int64_t> count(nrow, 0);
  const bool df = diag_first != 0;
  // pass 1: distinct columns per row -> indptr
  if (!over_rows(nrow, nthreads, [&](int64_t a, int64_t b) {
        return build_rows(cdofs, ndt, ndr, ncol, df, ri, a, b, count.data(), nullptr, nullptr,
                          nullptr);
      }))
    return HM_ERR_RANGE;
  int64_t acc = 0;
  indptr[0] = 0;
  for (int64_t r = 0; r < nrow; ++r) {
    acc += count[r];
    if (acc > INT32_MAX) return HM_ERR_UNSUPPORTED;
    indptr[r + 1] = (int32_t)acc;
  }
  *nnz = acc;
  if (!indices) return HM_OK;
  if (indices_capacity < acc) return HM_ERR_NOMEM;
  // pass 2: columns and entry positions at their final places
  if (!over_rows(nrow, nthreads, [&](int64_t a, int64_t b) {
        return build_rows(cdofs, ndt, ndr, ncol, df, ri, a, b, count.data(), indptr, indices, slot);
      }))
    return HM_ERR_RANGE;
  return HM_OK;
}
