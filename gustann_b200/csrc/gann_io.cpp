// Readers for the reference's index files, with the checks the reference
// leaves to assert()/exit() (src/layout.cpp, src/pq_search.cu, src/nav_graph.cu).
#include <cinttypes>
#include <cstdio>
#include <cstring>
#include <memory>
#include <string>

#include "gann_internal.h"

namespace gann {

namespace {

struct File {
  FILE* f = nullptr;
  explicit File(const std::string& path, const char* mode = "rb") { f = std::fopen(path.c_str(), mode); }
  ~File() {
    if (f) std::fclose(f);
  }
};

[[noreturn]] void fail(int code, const std::string& msg) { throw GannError{code, msg}; }

int64_t file_size(FILE* f) {
  long cur = std::ftell(f);
  std::fseek(f, 0, SEEK_END);
  int64_t sz = std::ftell(f);
  std::fseek(f, cur, SEEK_SET);
  return sz;
}

// DiskANN ".bin" block: int32 rows, int32 cols, rows*cols items
// (read_bin, src/pq_search.cu:187-201).
template <class T>
void read_bin_block(const std::string& path, int64_t offset, int& rows, int& cols, std::vector<T>& out) {
  File fl(path);
  if (!fl.f) fail(GANN_EIO, "cannot open " + path);
  int64_t size = file_size(fl.f);
  if (offset < 0 || offset + 8 > size || std::fseek(fl.f, (long)offset, SEEK_SET) != 0)
    fail(GANN_EFORMAT, "block offset outside " + path);
  if (std::fread(&rows, 4, 1, fl.f) != 1 || std::fread(&cols, 4, 1, fl.f) != 1 || rows < 0 || cols < 0)
    fail(GANN_EFORMAT, "bad block header in " + path);
  int64_t count = (int64_t)rows * cols;
  if (offset + 8 + count * (int64_t)sizeof(T) > size) fail(GANN_EIO, "short block in " + path);
  out.resize((size_t)count);
  if (count && std::fread(out.data(), sizeof(T), (size_t)count, fl.f) != (size_t)count)
    fail(GANN_EIO, "short read in " + path);
}

}  // namespace

// Header sector of DiskANN's _disk.index: uint32 nr, uint32 nc, then uint64
// n, dim, medoid, max_node_len, nodes_per_sector, ... (Layout::parse_diskann_metadata,
// src/layout.cpp:25-54); max_m0 = (max_node_len - dim*elt)/4 - 1 (layout.cpp:46).
void read_disk_index(const std::string& path, HostIndex& hx, std::vector<uint8_t>* pages_out) {
  File fl(path);
  if (!fl.f) fail(GANN_EIO, "cannot open index file " + path);
  uint32_t nr = 0, nc = 0;
  uint64_t v[5];
  if (std::fread(&nr, 4, 1, fl.f) != 1 || std::fread(&nc, 4, 1, fl.f) != 1 || std::fread(v, 8, 5, fl.f) != 5)
    fail(GANN_EFORMAT, "short header in " + path);
  if (nr < 5 || nc != 1) fail(GANN_EFORMAT, "index header is not a (>=5) x 1 metadata block: " + path);
  hx.n = (int64_t)v[0];
  hx.dim = (int64_t)v[1];
  hx.medoid = (int64_t)v[2];
  hx.node_len = (int64_t)v[3];
  hx.npp = (int64_t)v[4];
  hx.data_len = hx.dim * hx.elt;
  if (hx.n <= 0 || hx.n > INT32_MAX || hx.dim <= 0 || hx.dim > 4096)
    fail(GANN_EFORMAT, "index point count or dimension out of range: " + path);
  if (hx.node_len <= hx.data_len + 4 || hx.node_len > kPageSize || (hx.node_len - hx.data_len) % 4 != 0)
    fail(GANN_EFORMAT, "index node length inconsistent with dimension: " + path);
  hx.max_m0 = (hx.node_len - hx.data_len) / 4 - 1;
  if (hx.npp <= 0 || hx.npp * hx.node_len > kPageSize)
    fail(GANN_EFORMAT, "nodes per page inconsistent with node length: " + path);
  if (hx.data_len % 4 != 0)
    fail(GANN_EFORMAT, "vector bytes per node must be a multiple of 4 (aligned degree word): " + path);
  if (hx.medoid < 0 || hx.medoid >= hx.n) fail(GANN_EFORMAT, "medoid out of range: " + path);
  hx.num_pages = (hx.n + hx.npp - 1) / hx.npp;
  int64_t need = (int64_t)kPageSize * (hx.num_pages + 1);
  if (file_size(fl.f) < need) fail(GANN_EIO, "index file shorter than its pages: " + path);
  if (pages_out) {
    pages_out->resize((size_t)hx.num_pages * kPageSize);
    std::fseek(fl.f, kPageSize, SEEK_SET);
    if (std::fread(pages_out->data(), 1, pages_out->size(), fl.f) != pages_out->size())
      fail(GANN_EIO, "short read of index pages: " + path);
  }
}

// PQSearch::read_data, src/pq_search.cu:56-121.
void read_pq(const std::string& prefix, HostIndex& hx, std::vector<uint8_t>& codes) {
  const std::string piv = prefix + "_pivots.bin", cmp = prefix + "_compressed.bin";
  int rows, cols;
  read_bin_block<uint8_t>(cmp, 0, rows, cols, codes);
  if (rows != hx.n) fail(GANN_EFORMAT, "PQ code count differs from the index point count: " + cmp);
  if (cols <= 0 || cols > 256) fail(GANN_EFORMAT, "PQ chunk count out of range: " + cmp);
  hx.pq_m = cols;
  std::vector<uint64_t> offs;
  read_bin_block<uint64_t>(piv, 0, rows, cols, offs);
  if (!((rows == 4 || rows == 5) && cols == 1))  // pq_search.cu:77-79
    fail(GANN_EFORMAT, "PQ offsets table must be 4x1 or 5x1: " + piv);
  const bool legacy = rows == 5;
  read_bin_block<float>(piv, (int64_t)offs[0], rows, cols, hx.pivots);
  if (rows != kPivots || cols != hx.dim) fail(GANN_EFORMAT, "PQ pivots must be 256 x dim: " + piv);
  read_bin_block<float>(piv, (int64_t)offs[1], rows, cols, hx.centroid);
  if (rows != hx.dim || cols != 1) fail(GANN_EFORMAT, "PQ centroid must be dim x 1: " + piv);
  read_bin_block<int32_t>(piv, (int64_t)offs[legacy ? 3 : 2], rows, cols, hx.chunk_offsets);
  if (rows != hx.pq_m + 1 || cols != 1) fail(GANN_EFORMAT, "PQ chunk offsets must be (M+1) x 1: " + piv);
  // The reference maps each dimension to its chunk (pq_search.cu:108-115) and
  // indexes the table with chunk_id[i] (pq.cuh:36), so the ranges must tile [0, dim).
  if (hx.chunk_offsets[0] != 0 || hx.chunk_offsets[hx.pq_m] != hx.dim)
    fail(GANN_EFORMAT, "PQ chunk offsets must start at 0 and end at dim: " + piv);
  for (int c = 0; c < hx.pq_m; c++)
    if (hx.chunk_offsets[c + 1] <= hx.chunk_offsets[c])
      fail(GANN_EFORMAT, "PQ chunk offsets must be strictly increasing: " + piv);
}

// NavGraph::init, src/nav_graph.cu:41-100.
void read_nav(const std::string& dir, HostIndex& hx) {
  const std::string pidx = dir + "/nav_index", pdat = dir + "/nav_index.data", pmap = dir + "/map.txt";
  {
    File fl(pdat);
    if (!fl.f) fail(GANN_EIO, "cannot open " + pdat);
    int n = 0, d = 0;
    if (std::fread(&n, 4, 1, fl.f) != 1 || std::fread(&d, 4, 1, fl.f) != 1 || n <= 0)
      fail(GANN_EFORMAT, "bad header in " + pdat);
    if (d != hx.dim) fail(GANN_EFORMAT, "pivot-graph vectors have a different dimension: " + pdat);
    hx.nav_n = n;
    hx.nav_data.resize((size_t)n * d * hx.elt);
    if (std::fread(hx.nav_data.data(), 1, hx.nav_data.size(), fl.f) != hx.nav_data.size())
      fail(GANN_EIO, "short read in " + pdat);
  }
  {
    File fl(pmap, "r");
    if (!fl.f) fail(GANN_EIO, "cannot open " + pmap);
    hx.nav_map.resize(hx.nav_n);
    for (int i = 0; i < hx.nav_n; i++) {
      int x;
      if (std::fscanf(fl.f, "%d", &x) != 1) fail(GANN_EFORMAT, "map.txt has fewer ids than pivot points");
      if (x < 0 || x >= hx.n) fail(GANN_EFORMAT, "map.txt id outside the index");
      hx.nav_map[i] = x;
    }
  }
  {
    File fl(pidx);
    if (!fl.f) fail(GANN_EIO, "cannot open " + pidx);
    int32_t hdr[6];  // u64 size, u32 max degree, u32 start, u64 frozen (nav_graph.cu:75-81)
    if (std::fread(hdr, 4, 6, fl.f) != 6) fail(GANN_EFORMAT, "short header in " + pidx);
    hx.nav_max_m = hdr[2];
    hx.nav_start = hdr[3];
    if (!(hx.nav_max_m > 0 && hx.nav_max_m <= 32))  // nav_graph.cu:84
      fail(GANN_EFORMAT, "pivot-graph max degree must be in 1..32: " + pidx);
    if (hx.nav_start < 0 || hx.nav_start >= hx.nav_n) fail(GANN_EFORMAT, "pivot-graph start out of range");
    hx.nav_graph.assign((size_t)hx.nav_n * hx.nav_max_m, -1);
    for (int i = 0; i < hx.nav_n; i++) {
      int32_t d;
      if (std::fread(&d, 4, 1, fl.f) != 1 || d <= 0 || d > hx.nav_max_m)  // nav_graph.cu:88
        fail(GANN_EFORMAT, "bad pivot-graph degree in " + pidx);
      int32_t* row = hx.nav_graph.data() + (size_t)i * hx.nav_max_m;
      if (std::fread(row, 4, (size_t)d, fl.f) != (size_t)d) fail(GANN_EIO, "short read in " + pidx);
      for (int j = 0; j < d; j++)
        if (row[j] < 0 || row[j] >= hx.nav_n) fail(GANN_EFORMAT, "pivot-graph neighbour out of range");
    }
  }
  hx.has_nav = true;
}

}  // namespace gann
