// Graph loaders with the reference loader's exact semantics, so that a file
// loaded here yields the same CSR as puercgp_examples::load_matrix_market /
// load_binary_csr_directory (puercgp/examples/mtx_loader.hxx:99-260).
#include <algorithm>
#include <cctype>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <sstream>
#include <string>
#include <tuple>
#include <vector>

#include "cgp_b200_internal.h"

namespace {

bool alloc_csr(cgp_host_csr* out, int64_t V, int64_t E) {
  std::memset(out, 0, sizeof(*out));
  out->num_vertices = V;
  out->num_edges = E;
  out->row_offsets = static_cast<int64_t*>(std::malloc(sizeof(int64_t) * (V + 1)));
  out->col_indices = static_cast<int32_t*>(std::malloc(sizeof(int32_t) * (E > 0 ? E : 1)));
  out->weights = std::malloc(sizeof(float) * (E > 0 ? E : 1));
  out->weight_kind = CGP_WEIGHT_F32;
  if (!out->row_offsets || !out->col_indices || !out->weights) {
    cgp_host_csr_free(out);
    return false;
  }
  return true;
}

std::string lower(std::string s) {
  for (char& c : s) c = static_cast<char>(std::tolower(static_cast<unsigned char>(c)));
  return s;
}

}  // namespace

extern "C" {

// Matrix Market coordinate files: 1-based (row, col[, value]) entries;
// "pattern" files get weight 1; "symmetric" files add the mirrored entry for
// every off-diagonal one; entries are sorted by (src, dst, weight) and kept
// as they are (duplicates and self loops included), as the reference does.
cgp_status cgp_load_matrix_market(const char* path, cgp_host_csr* out) {
  cgp::clear_error();
  if (path == nullptr || out == nullptr) return cgp::set_error(CGP_ERR_INVALID_ARG, "NULL argument");
  std::memset(out, 0, sizeof(*out));
  std::ifstream in(path);
  if (!in) return cgp::set_error(CGP_ERR_INVALID_ARG, std::string("could not open matrix: ") + path);
  std::string header;
  std::getline(in, header);
  const std::string hl = lower(header);
  const bool pattern = hl.find("pattern") != std::string::npos;
  const bool symmetric = hl.find("symmetric") != std::string::npos;
  std::string line;
  do {
    if (!std::getline(in, line))
      return cgp::set_error(CGP_ERR_INVALID_ARG, std::string("missing matrix dimensions: ") + path);
  } while (line.empty() || line[0] == '%');
  long long rows = 0, cols = 0, entries = 0;
  {
    std::istringstream dims(line);
    dims >> rows >> cols >> entries;
  }
  const int64_t V = std::max(rows, cols);
  if (V <= 0 || V >= INT32_MAX || entries < 0)
    return cgp::set_error(CGP_ERR_INVALID_ARG, "bad matrix dimensions");
  std::vector<std::tuple<int32_t, int32_t, float>> edges;
  edges.reserve(static_cast<size_t>(entries) * (symmetric ? 2 : 1));
  for (long long i = 0; i < entries; ++i) {
    if (!std::getline(in, line))
      return cgp::set_error(CGP_ERR_INVALID_ARG, std::string("truncated matrix: ") + path);
    if (line.empty() || line[0] == '%') {
      --i;
      continue;
    }
    std::istringstream row(line);
    long long s = 0, d = 0;
    float w = 1.0f;
    row >> s >> d;
    if (!pattern) row >> w;
    --s;
    --d;
    if (s < 0 || s >= V || d < 0 || d >= V)
      return cgp::set_error(CGP_ERR_INVALID_ARG, std::string("vertex out of range in: ") + path);
    edges.emplace_back(static_cast<int32_t>(s), static_cast<int32_t>(d), w);
    if (symmetric && s != d) edges.emplace_back(static_cast<int32_t>(d), static_cast<int32_t>(s), w);
  }
  std::sort(edges.begin(), edges.end());
  const int64_t E = static_cast<int64_t>(edges.size());
  if (!alloc_csr(out, V, E)) return cgp::set_error(CGP_ERR_OOM, "host allocation failed");
  std::vector<int64_t> deg(V + 1, 0);
  for (const auto& t : edges) ++deg[std::get<0>(t) + 1];
  out->row_offsets[0] = 0;
  for (int64_t v = 0; v < V; ++v) out->row_offsets[v + 1] = out->row_offsets[v] + deg[v + 1];
  float* w = static_cast<float*>(out->weights);
  for (int64_t e = 0; e < E; ++e) {  // edges are sorted by source, so positions are in order
    out->col_indices[e] = std::get<1>(edges[e]);
    w[e] = std::get<2>(edges[e]);
  }
  return CGP_OK;
}

// Directory with csr_vlist.bin (int32 offsets), csr_elist.bin (int32
// columns) and optionally csr_weightlist.bin (int32 weights, read as float);
// without the weight file every weight is 1.
cgp_status cgp_load_binary_csr(const char* dir, cgp_host_csr* out) {
  cgp::clear_error();
  if (dir == nullptr || out == nullptr) return cgp::set_error(CGP_ERR_INVALID_ARG, "NULL argument");
  std::memset(out, 0, sizeof(*out));
  const std::string base(dir);
  auto read_all = [](const std::string& p, std::vector<int32_t>& v) -> int {
    FILE* f = std::fopen(p.c_str(), "rb");
    if (!f) return 1;
    std::fseek(f, 0, SEEK_END);
    long n = std::ftell(f);
    std::fseek(f, 0, SEEK_SET);
    if (n < 0 || n % 4 != 0) {
      std::fclose(f);
      return 2;
    }
    v.resize(static_cast<size_t>(n) / 4);
    size_t got = v.empty() ? 0 : std::fread(v.data(), 4, v.size(), f);
    std::fclose(f);
    return got == v.size() ? 0 : 3;
  };
  std::vector<int32_t> row, col, wt;
  if (read_all(base + "/csr_vlist.bin", row) != 0 || read_all(base + "/csr_elist.bin", col) != 0)
    return cgp::set_error(CGP_ERR_INVALID_ARG,
                          "CSR directory must contain csr_vlist.bin and csr_elist.bin of 32-bit integers: " + base);
  if (row.size() < 2) return cgp::set_error(CGP_ERR_INVALID_ARG, "csr_vlist.bin too short");
  const int64_t V = static_cast<int64_t>(row.size()) - 1;
  const int64_t E = static_cast<int64_t>(col.size());
  int wr = read_all(base + "/csr_weightlist.bin", wt);
  const bool has_w = wr == 0;
  if (wr != 1 && wr != 0) return cgp::set_error(CGP_ERR_INVALID_ARG, "bad csr_weightlist.bin");
  if (has_w && wt.size() != col.size())
    return cgp::set_error(CGP_ERR_INVALID_ARG, "csr_weightlist.bin size must equal csr_elist.bin size");
  if (!alloc_csr(out, V, E)) return cgp::set_error(CGP_ERR_OOM, "host allocation failed");
  for (int64_t v = 0; v <= V; ++v) out->row_offsets[v] = row[v];
  std::memcpy(out->col_indices, col.data(), sizeof(int32_t) * E);
  float* w = static_cast<float*>(out->weights);
  for (int64_t e = 0; e < E; ++e) w[e] = has_w ? static_cast<float>(wt[e]) : 1.0f;
  return CGP_OK;
}

// Galois binary graph, version 1 (the reader of cgp/examples/algorithms/bfs/
// cgp_bfs.cu:215-260): four uint64 header words (version = 1, bytes of edge
// data per edge, vertex count V, edge count E), V uint64 row ends, E uint32
// destinations, padding to 8 bytes when E is odd, then E edge-data records.
// The reference loader reads the topology only (unit weights); with
// read_edge_data != 0 and 4-byte edge data the records are kept as uint32
// weights.  Truncated files, other versions, sizes beyond int32 vertex ids,
// decreasing row ends and destinations outside [0, V) are rejected.
cgp_status cgp_load_galois_gr(const char* path, int32_t read_edge_data, cgp_host_csr* out) {
  cgp::clear_error();
  if (path == nullptr || out == nullptr) return cgp::set_error(CGP_ERR_INVALID_ARG, "NULL argument");
  std::memset(out, 0, sizeof(*out));
  FILE* f = std::fopen(path, "rb");
  if (!f) return cgp::set_error(CGP_ERR_INVALID_ARG, std::string("could not open graph: ") + path);
  auto fail = [&](const std::string& m) {
    std::fclose(f);
    cgp_host_csr_free(out);
    return cgp::set_error(CGP_ERR_INVALID_ARG, m + ": " + path);
  };
  uint64_t hdr[4];
  if (std::fread(hdr, sizeof(uint64_t), 4, f) != 4) return fail("truncated .gr header");
  const uint64_t version = hdr[0], edge_bytes = hdr[1], V64 = hdr[2], E64 = hdr[3];
  if (version != 1) return fail("unsupported .gr version " + std::to_string(version));
  if (V64 == 0 || V64 >= static_cast<uint64_t>(INT32_MAX))
    return fail(".gr vertex count must be in [1, 2^31-1)");
  if (E64 > (static_cast<uint64_t>(1) << 40)) return fail(".gr edge count too large");
  const int64_t V = static_cast<int64_t>(V64), E = static_cast<int64_t>(E64);
  out->num_vertices = V;
  out->num_edges = E;
  out->row_offsets = static_cast<int64_t*>(std::malloc(sizeof(int64_t) * (V + 1)));
  out->col_indices = static_cast<int32_t*>(std::malloc(sizeof(int32_t) * (E > 0 ? E : 1)));
  if (!out->row_offsets || !out->col_indices) {
    std::fclose(f);
    cgp_host_csr_free(out);
    return cgp::set_error(CGP_ERR_OOM, "host allocation failed");
  }
  out->row_offsets[0] = 0;
  if (std::fread(out->row_offsets + 1, sizeof(int64_t), V, f) != static_cast<size_t>(V))
    return fail("truncated .gr row ends");
  for (int64_t v = 0; v < V; ++v)
    if (out->row_offsets[v + 1] < out->row_offsets[v]) return fail(".gr row ends decrease");
  if (out->row_offsets[V] != E) return fail(".gr final row end does not match the edge count");
  if (E > 0 && std::fread(out->col_indices, sizeof(int32_t), E, f) != static_cast<size_t>(E))
    return fail("truncated .gr destinations");
  for (int64_t e = 0; e < E; ++e)
    if (out->col_indices[e] < 0 || out->col_indices[e] >= V)
      return fail(".gr destination out of range at edge " + std::to_string(e));
  if (read_edge_data && edge_bytes == 4 && E > 0) {
    if (E % 2 == 1) {
      uint32_t pad;
      if (std::fread(&pad, 4, 1, f) != 1) return fail("truncated .gr padding");
    }
    out->weights = std::malloc(sizeof(uint32_t) * E);
    if (!out->weights) {
      std::fclose(f);
      cgp_host_csr_free(out);
      return cgp::set_error(CGP_ERR_OOM, "host allocation failed");
    }
    if (std::fread(out->weights, sizeof(uint32_t), E, f) != static_cast<size_t>(E))
      return fail("truncated .gr edge data");
    out->weight_kind = CGP_WEIGHT_U32;
  } else if (read_edge_data && edge_bytes != 0 && edge_bytes != 4) {
    return fail(".gr edge data of " + std::to_string(edge_bytes) + " bytes cannot be read as weights");
  }
  std::fclose(f);
  return CGP_OK;
}

}  // extern "C"
