// The FlashGraph 1D format: a graph image (graph_header page plus vertex
// records) turned into the host CSR that the SpMM scheduler takes.
//
//   header  flash-graph/graph_file_header.h:27-37 (one 4096-byte page):
//           int64 magic 0x123456789ABCDEF, int32 version 4, int32 type
//           (DIRECTED 0, UNDIRECTED 1, TS_DIRECTED 2, TS_UNDIRECTED 3),
//           uint64 num_vertices, uint64 num_edges, int32 edge_data_size,
//           int32 max_num_timestamps
//   record  ext_mem_undirected_vertex (flash-graph/vertex.h:444-562):
//           uint32 id, uint32 edge_data_size, uint32 num_edges, uint32
//           neighbors[num_edges]; edge data at round_up(12 + 4 num_edges,
//           edge_data_size), the record then rounded up to 4 bytes
//           (round_up(off, b) = (off + b - 1) & ~(b - 1), libsafs/common_c.h:36)
//   file    mem_directed_graph::dump_graph (flash-graph/utils.cpp:399-420):
//           all in-edge records, then all out-edge records; an undirected
//           graph has one record per vertex
#include "fmx_internal.h"

#include <cstdio>
#include <new>

namespace fmx {
namespace {

constexpr int64_t kFgMagic = 0x123456789ABCDEFLL;
constexpr int kFgVersion = 4;

struct fg_header {
	int64_t magic;
	int32_t version, type;
	uint64_t num_vertices, num_edges;
	int32_t edge_data_size, max_num_timestamps;
};
static_assert(sizeof(fg_header) == 40, "graph_header_struct layout (x86-64)");

uint64_t round_up(uint64_t off, uint64_t base) { return (off + base - 1) & ~(base - 1); }
uint64_t data_off(uint32_t ne, uint32_t eds) { return eds ? round_up(12 + 4ull * ne, eds) : 12 + 4ull * ne; }
uint64_t record_size(uint32_t ne, uint32_t eds)
{
	return eds ? round_up(data_off(ne, eds) + uint64_t(ne) * eds, 4) : 12 + 4ull * ne;
}

// Walk one part's n records from `at`: the CSR of that part (if `out`), and
// the offset after its last record.
int walk_part(const char *b, size_t len, uint64_t &at, uint64_t n, uint32_t eds, int prim, host_csr *out)
{
	std::vector<uint64_t> starts;
	if (out) {
		out->nrows = out->ncols = n;
		out->prim = prim;
		out->esize = eds;
		out->row_ptr.assign(n + 1, 0);
		starts.resize(n);
	}
	uint64_t nnz = 0;
	for (uint64_t v = 0; v < n; v++) {
		uint32_t r[3];
		if (at + 12 > len) return set_error(FMX_ERR_IMAGE, "graph image ends inside vertex %llu's record", (unsigned long long)v);
		memcpy(r, b + at, 12);
		if (r[0] != v)
			return set_error(FMX_ERR_IMAGE, "record %llu names vertex %u (records must be in id order)",
					(unsigned long long)v, r[0]);
		if (r[1] != eds)
			return set_error(FMX_ERR_IMAGE, "vertex %u has %u bytes of edge data, the header %u", r[0], r[1], eds);
		const uint64_t sz = record_size(r[2], eds);
		if (at + sz > len) return set_error(FMX_ERR_IMAGE, "vertex %u's record runs past the image", r[0]);
		if (out) {
			starts[v] = at;
			nnz += r[2];
			if (nnz >= (1ull << 32)) return set_error(FMX_ERR_UNSUPPORTED, "more than 2^32 edges in one part");
			out->row_ptr[v + 1] = uint32_t(nnz);
		}
		at += sz;
	}
	if (!out) return FMX_OK;
	out->nnz = nnz;
	out->col.resize(nnz);
	out->val.resize(nnz * eds);
	for (uint64_t v = 0; v < n; v++) {
		uint32_t ne;
		memcpy(&ne, b + starts[v] + 8, 4);
		const uint64_t o = out->row_ptr[v];
		for (uint32_t i = 0; i < ne; i++) {
			uint32_t c;
			memcpy(&c, b + starts[v] + 12 + 4ull * i, 4);
			if (c >= n) return set_error(FMX_ERR_IMAGE, "vertex %llu has neighbor %u of %llu vertices",
					(unsigned long long)v, c, (unsigned long long)n);
			out->col[o + i] = int32_t(c);
		}
		if (eds) memcpy(out->val.data() + o * eds, b + starts[v] + data_off(ne, eds), size_t(ne) * eds);
	}
	return FMX_OK;
}

} // namespace
} // namespace fmx

using namespace fmx;

extern "C" {

int fmx_matrix_from_fg(const void *adj, size_t adj_len, int val_type, int device, fmx_matrix **out)
{
	if (!adj || !out) return set_error(FMX_ERR_INVAL, "null argument");
	*out = nullptr;
	const char *b = static_cast<const char *>(adj);
	if (adj_len < kPage) return set_error(FMX_ERR_IMAGE, "a graph image starts with a %zu-byte header page", kPage);
	fg_header h;
	memcpy(&h, b, sizeof(h));
	if (h.magic != kFgMagic) return set_error(FMX_ERR_IMAGE, "not a FlashGraph graph image (magic %llx)",
			(unsigned long long)h.magic);
	if (h.version != kFgVersion) return set_error(FMX_ERR_IMAGE, "graph image version %d, expected %d", h.version, kFgVersion);
	if (h.type == 2 || h.type == 3) return set_error(FMX_ERR_UNSUPPORTED, "time-series graphs have no sparse matrix form");
	if (h.type != 0 && h.type != 1) return set_error(FMX_ERR_IMAGE, "unknown graph type %d", h.type);
	if (h.edge_data_size < 0) return set_error(FMX_ERR_IMAGE, "negative edge data size");
	const uint32_t eds = uint32_t(h.edge_data_size);
	const size_t want = prim_size(val_type);
	if (want == size_t(-1)) return set_error(FMX_ERR_TYPE, "unknown value type %d", val_type);
	if (want != eds)
		return set_error(FMX_ERR_TYPE, "the graph has %u bytes of edge data per edge; value type %d has %zu", eds,
				val_type, want);
	if (h.num_vertices >= (1ull << 31)) return set_error(FMX_ERR_UNSUPPORTED, "%llu vertices exceed int32 indices",
			(unsigned long long)h.num_vertices);
	const bool directed = h.type == 0;
	int rc;
	try {
		uint64_t at = kPage;
		host_csr a, t;
		if (directed) {
			rc = walk_part(b, adj_len, at, h.num_vertices, eds, val_type, &t);          // in-edge records: A^T
			if (!rc) rc = walk_part(b, adj_len, at, h.num_vertices, eds, val_type, &a); // out-edge records: A
		} else {
			rc = walk_part(b, adj_len, at, h.num_vertices, eds, val_type, &a);
		}
		if (!rc) rc = matrix_from_csr(a, directed ? &t : nullptr, device, out);
	} catch (const std::bad_alloc &) {
		rc = set_error(FMX_ERR_OOM, "host allocation failed while reading the graph image");
	}
	return rc;
}

int fmx_matrix_load_fg(const char *adj_path, int val_type, int device, fmx_matrix **out)
{
	if (!adj_path || !out) return set_error(FMX_ERR_INVAL, "null argument");
	*out = nullptr;
	FILE *f = fopen(adj_path, "rb");
	if (!f) return set_error(FMX_ERR_IO, "cannot open %s", adj_path);
	std::vector<char> buf;
	int rc = FMX_OK;
	try {
		if (fseeko(f, 0, SEEK_END) != 0) rc = set_error(FMX_ERR_IO, "cannot seek %s", adj_path);
		const off_t len = rc ? 0 : ftello(f);
		if (!rc && len < 0) rc = set_error(FMX_ERR_IO, "cannot size %s", adj_path);
		if (!rc) {
			buf.resize(size_t(len));
			fseeko(f, 0, SEEK_SET);
			if (len && fread(buf.data(), 1, size_t(len), f) != size_t(len)) rc = set_error(FMX_ERR_IO, "short read of %s", adj_path);
		}
	} catch (const std::bad_alloc &) {
		rc = set_error(FMX_ERR_OOM, "no host memory for %s", adj_path);
	}
	fclose(f);
	if (rc) return rc;
	return fmx_matrix_from_fg(buf.data(), buf.size(), val_type, device, out);
}

} // extern "C"
