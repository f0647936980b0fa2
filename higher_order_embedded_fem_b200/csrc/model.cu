// Model setup: shared CSR pattern, greedy colorings and element-to-nnz maps.
//
// Reference: CsrParAssembler::assemble_pattern (fenris/src/assembly.rs:177-249),
// CooMatrix::to_csr (fenris/src/sparse.rs:102-165), color_nodes /
// sequential_greedy_coloring (fenris/src/assembly.rs:1403-1411,
// paradis/src/coloring.rs:48-72), NodalModel / EmbeddedModel construction
// (fenris/src/model.rs:90-117, fenris/src/embedding/mod.rs:243-283).
//
// The pattern of a vector-valued (3 components) FE matrix is fully described
// by the node adjacency: row 3a+i holds the columns 3b+j of every node b that
// shares an element with a, in ascending order.  It is stored as the sorted
// adjacency lists plus base[a] = row_offsets[3a]; the explicit row offsets and
// column indices the reference uses are produced from it on request and are
// identical to the reference's (sorted, de-duplicated coordinates).
#include <algorithm>
#include <cstring>
#include <numeric>

#include "internal.h"

namespace hoefem {

BlockDev Block::dev() const {
  BlockDev b;
  b.kind = kind;
  b.nn = nn;
  b.ne = (int)ne;
  b.conn = d_conn.p;
  b.uniform = uniform ? 1 : 0;
  b.nq = uniform ? (int)qw.size() : 0;
  b.qoff = uniform ? nullptr : d_qoff.p;
  b.qw = d_qw.p;
  b.qp = d_qp.p;
  b.emap = d_emap.p;
  b.emat = d_emat.p;
  b.escene = d_escene.p;
  b.scene_active = d_escene.p ? scene_active : nullptr;
  return b;
}

NodeRows Model::rows() const {
  NodeRows r;
  r.nv = (int)nv;
  r.base = d_base.p;
  r.adj_off = d_adj_off.p;
  r.adj = d_adj.p;
  r.diag_slot = d_diag_slot.p;
  r.diag_only = nullptr;
  r.lanes = spmv_lanes;
  r.sched = d_sched.p;
  return r;
}

Model::~Model() {
  for (Block* b : blocks) delete b;
  if (stream) cudaStreamDestroy(stream);
}

// First-fit greedy coloring identical to paradis' sequential_greedy_coloring:
// an element joins the first existing color none of whose elements shares a
// node with it, otherwise opens a new color.  Per node a bitset of the colors
// that already contain it makes the test O(nodes * words).
void greedy_coloring(const i64* conn, i64 ne, int nn, i64 nv, std::vector<i64>& color_off,
                     std::vector<int>& color_elems) {
  std::vector<std::vector<uint64_t>> used(nv);
  std::vector<int> color(ne);
  int ncolors = 0;
  std::vector<uint64_t> acc;
  for (i64 e = 0; e < ne; ++e) {
    const i64* c = conn + e * nn;
    int words = (ncolors + 63) / 64;
    acc.assign(words + 1, 0);
    for (int I = 0; I < nn; ++I) {
      const auto& u = used[c[I]];
      for (size_t w = 0; w < u.size(); ++w) acc[w] |= u[w];
    }
    int col = 0;
    while (col < ncolors && ((acc[col >> 6] >> (col & 63)) & 1ull)) ++col;
    if (col == ncolors) ++ncolors;
    color[e] = col;
    for (int I = 0; I < nn; ++I) {
      auto& u = used[c[I]];
      if ((int)u.size() <= (col >> 6)) u.resize((col >> 6) + 1, 0);
      u[col >> 6] |= 1ull << (col & 63);
    }
  }
  color_off.assign(ncolors + 1, 0);
  for (i64 e = 0; e < ne; ++e) color_off[color[e] + 1]++;
  for (int k = 0; k < ncolors; ++k) color_off[k + 1] += color_off[k];
  color_elems.resize(ne);
  std::vector<i64> fill(color_off.begin(), color_off.end() - 1);
  for (i64 e = 0; e < ne; ++e) color_elems[fill[color[e]]++] = (int)e;
}

// Sorted, de-duplicated neighbour lists of every node over a set of ragged
// node lists (elements or Schwarz subdomains).
void node_adjacency(i64 nv, const std::vector<const std::vector<i64>*>& conns, const std::vector<int>& nns,
                    std::vector<int>& adj_off, std::vector<int>& adj) {
  std::vector<i64> cnt(nv + 1, 0);
  for (size_t b = 0; b < conns.size(); ++b) {
    const auto& c = *conns[b];
    int nn = nns[b];
    i64 ne = nn ? (i64)c.size() / nn : 0;
    for (i64 e = 0; e < ne; ++e)
      for (int I = 0; I < nn; ++I) cnt[c[e * nn + I] + 1] += nn;
  }
  for (i64 a = 0; a < nv; ++a) cnt[a + 1] += cnt[a];
  std::vector<int> tmp(cnt[nv]);
  std::vector<i64> pos(cnt.begin(), cnt.end() - 1);
  for (size_t b = 0; b < conns.size(); ++b) {
    const auto& c = *conns[b];
    int nn = nns[b];
    i64 ne = nn ? (i64)c.size() / nn : 0;
    for (i64 e = 0; e < ne; ++e)
      for (int I = 0; I < nn; ++I) {
        i64 a = c[e * nn + I];
        for (int J = 0; J < nn; ++J) tmp[pos[a]++] = (int)c[e * nn + J];
      }
  }
  adj_off.assign(nv + 1, 0);
  adj.clear();
  adj.reserve(tmp.size() / 4);
  for (i64 a = 0; a < nv; ++a) {
    auto b = tmp.begin() + cnt[a], en = tmp.begin() + cnt[a + 1];
    std::sort(b, en);
    auto last = std::unique(b, en);
    adj.insert(adj.end(), b, last);
    adj_off[a + 1] = (int)adj.size();
  }
}

static void build_emap(const Block& blk, const std::vector<int>& adj_off, const std::vector<int>& adj,
                       const std::vector<long long>& base, std::vector<int>& emap) {
  const int nn = blk.nn;
  emap.resize((size_t)blk.ne * nn * nn);
  for (i64 e = 0; e < blk.ne; ++e) {
    const i64* c = blk.conn.data() + e * nn;
    for (int I = 0; I < nn; ++I) {
      i64 a = c[I];
      const int* b0 = adj.data() + adj_off[a];
      const int* b1 = adj.data() + adj_off[a + 1];
      for (int J = 0; J < nn; ++J) {
        const int* it = std::lower_bound(b0, b1, (int)c[J]);
        HOEFEM_REQUIRE(it != b1 && *it == (int)c[J], HOEFEM_ERR_PATTERN, "element node missing from pattern");
        emap[(size_t)e * nn * nn + I * nn + J] = (int)(3 * (it - b0));
      }
    }
  }
}

void finalize_model(Model& m) {
  HOEFEM_REQUIRE(!m.finalized, HOEFEM_ERR_INVALID_ARGUMENT, "model already finalized");
  HOEFEM_REQUIRE(!m.blocks.empty(), HOEFEM_ERR_INVALID_ARGUMENT, "model has no element block");
  std::vector<const std::vector<i64>*> conns;
  std::vector<int> nns;
  m.num_elements = 0;
  for (Block* b : m.blocks) {
    // An element that repeats a node cannot be scattered (the reference panics
    // in add_element_row_to_csr_row); reject it up front.
    for (i64 e = 0; e < b->ne; ++e) {
      i64 tmp[27];
      std::copy(b->conn.begin() + e * b->nn, b->conn.begin() + (e + 1) * b->nn, tmp);
      std::sort(tmp, tmp + b->nn);
      for (int k = 0; k + 1 < b->nn; ++k)
        HOEFEM_REQUIRE(tmp[k] != tmp[k + 1], HOEFEM_ERR_PATTERN, "element with repeated node");
      HOEFEM_REQUIRE(tmp[0] >= 0 && tmp[b->nn - 1] < m.nv, HOEFEM_ERR_INVALID_ARGUMENT, "node index out of range");
    }
    conns.push_back(&b->conn);
    nns.push_back(b->nn);
    m.num_elements += b->ne;
  }
  node_adjacency(m.nv, conns, nns, m.adj_off, m.adj);
  m.base.assign(m.nv + 1, 0);
  m.diag_slot.assign(m.nv, -1);
  for (i64 a = 0; a < m.nv; ++a) {
    i64 d = m.adj_off[a + 1] - m.adj_off[a];
    m.base[a + 1] = m.base[a] + 9 * d;
    const int* b0 = m.adj.data() + m.adj_off[a];
    const int* e0 = m.adj.data() + m.adj_off[a + 1];
    const int* it = std::lower_bound(b0, e0, (int)a);
    if (it != e0 && *it == a) m.diag_slot[a] = (int)(it - b0);
  }
  m.ndof = 3 * m.nv;
  m.nnz = m.base[m.nv];
  HOEFEM_REQUIRE(3 * m.nv < (i64)2147483647, HOEFEM_ERR_INVALID_ARGUMENT, "more than 2^31 DOFs");

  for (Block* b : m.blocks) greedy_coloring(b->conn.data(), b->ne, b->nn, m.nv, b->color_off, b->color_elems);
  m.finalized = true;
}

// Device copy of the model (created on first use, on the current device).
void ensure_device(Model& m) {
  HOEFEM_REQUIRE(m.finalized, HOEFEM_ERR_NOT_FINALIZED, "model is not finalized");
  if (m.on_device) return;
  int count = 0;
  if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) {
    cudaGetLastError();
    throw Error(HOEFEM_ERR_NO_DEVICE, "no CUDA device available");
  }
  HOEFEM_CUDA(cudaGetDevice(&m.device));
  if (!m.stream) HOEFEM_CUDA(cudaStreamCreateWithFlags(&m.stream, cudaStreamNonBlocking));
  cudaStream_t s = m.stream;
  m.d_X.upload(m.X, s);
  m.d_adj_off.upload(m.adj_off, s);
  m.d_adj.upload(m.adj, s);
  m.d_diag_slot.upload(m.diag_slot, s);
  m.d_base.upload(m.base, s);
  m.d_err.alloc(1);
  m.d_sched.alloc(2);
  m.d_sched.zero(s);
  m.d_err.zero(s);
  for (Block* b : m.blocks) {
    std::vector<int> soa((size_t)b->ne * b->nn);
    for (i64 e = 0; e < b->ne; ++e)
      for (int I = 0; I < b->nn; ++I) soa[(size_t)I * b->ne + e] = (int)b->conn[e * b->nn + I];
    b->d_conn.upload(soa, s);
    std::vector<int> emap;
    build_emap(*b, m.adj_off, m.adj, m.base, emap);
    b->d_emap.upload(emap, s);
    b->d_color_elems.upload(b->color_elems, s);
    b->d_qw.upload(b->qw, s);
    b->d_qp.upload(b->qp, s);
    if (!b->uniform) {
      std::vector<int> qo(b->qoff.begin(), b->qoff.end());
      b->d_qoff.upload(qo, s);
    }
    if (!b->emat.empty()) b->d_emat.upload(b->emat, s);
    if (!b->escene.empty()) b->d_escene.upload(b->escene, s);
  }
  HOEFEM_CUDA(cudaStreamSynchronize(s));
  m.on_device = true;
}

// Explicit row offsets / column indices (identical to the reference pattern).
void export_pattern(const std::vector<int>& adj_off, const std::vector<int>& adj, const std::vector<long long>& base,
                    const std::vector<unsigned char>* diag_only, i64 nv, int64_t* ro, int64_t* ci) {
  for (i64 a = 0; a < nv; ++a) {
    bool dg = diag_only && (*diag_only)[a];
    i64 d = adj_off[a + 1] - adj_off[a];
    for (int i = 0; i < 3; ++i) {
      i64 r = 3 * a + i;
      if (dg) {
        ro[r] = base[a] + i;
        ci[base[a] + i] = r;
      } else {
        ro[r] = base[a] + i * 3 * d;
        i64 k = ro[r];
        for (i64 s = 0; s < d; ++s)
          for (int j = 0; j < 3; ++j) ci[k++] = 3 * (i64)adj[adj_off[a] + s] + j;
      }
    }
  }
  ro[3 * nv] = base[nv];
}

void check_device_error(const Model& m) {
  int err = 0;
  HOEFEM_CUDA(cudaMemcpyAsync(&err, m.d_err.p, sizeof(int), cudaMemcpyDeviceToHost, m.stream));
  HOEFEM_CUDA(cudaStreamSynchronize(m.stream));
  if (err) {
    HOEFEM_CUDA(cudaMemsetAsync(m.d_err.p, 0, sizeof(int), m.stream));
    throw Error(err, err == HOEFEM_ERR_SINGULAR ? "singular Jacobian or deformation gradient in an element"
                                                : "device error");
  }
}

}  // namespace hoefem
