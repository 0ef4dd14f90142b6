/*
 * ref_fg_walk.cpp -- walks a FlashGraph adjacency image with FlashGraph's OWN
 * record and header classes.
 *
 * TEST INFRASTRUCTURE ONLY (the checker of the checker).  Built by
 * oracle/Makefile against the reference headers where they lie
 * (flash-graph/vertex.h, flash-graph/graph_file_header.h,
 * flash-graph/FG_basic_types.h, libsafs/common_c.h, libsafs/comm_exception.h)
 * into oracle/_ref/.  Nothing from the reference is copied into this
 * repository; the four SAFS headers that need Boost are replaced by the
 * stubs in oracle/ref_stubs_fg/.
 *
 * Record sizes, edge-data offsets, neighbor and edge-data reads use the
 * reference's inline methods (ext_mem_undirected_vertex::get_size,
 * num_edges2vsize, get_edge_data_offset, get_neighbor, get_edge_data,
 * graph_header accessors).  The per-row arithmetic restates
 * fg_row_spmm_task::run_on_row (flash-graph/fg_sparse_matrix.cpp:83-106),
 * which lives in a file that cannot be compiled here.
 */
#include <stdint.h>
#include <string.h>
#include <vector>
#include "graph_file_header.h"
#include "vertex.h"

using namespace fg;

template<class T, class S>
static int walk(const char *adj, uint64_t len, int transpose, const T *X, T *Y, uint64_t k)
{
	const graph_header *h = reinterpret_cast<const graph_header *>(adj);
	const uint64_t n = h->get_num_vertices();
	const bool directed = h->is_directed_graph();
	uint64_t at = graph_header::get_header_size();
	for (int part = 0; part < (directed ? 2 : 1); part++) {
		const bool use = !directed || ((part == 0) == (transpose != 0));
		for (uint64_t v = 0; v < n; v++) {
			const ext_mem_undirected_vertex *r = reinterpret_cast<const ext_mem_undirected_vertex *>(adj + at);
			if (at + ext_mem_undirected_vertex::get_header_size() > len || r->get_id() != v) return -1;
			if (at + r->get_size() > len) return -1;
			if (use) {
				std::vector<T> res(k, T(0));
				const bool has_val = r->has_edge_data();
				for (size_t i = 0; i < r->get_num_edges(); i++) {
					const vertex_id_t id = r->get_neighbor(i);
					if (id >= n) return -1;
					T data = 1;
					if (has_val) data = T(r->template get_edge_data<S>(i));
					const T *row = X + uint64_t(id) * k;
					for (size_t j = 0; j < k; j++) res[j] += row[j] * data;
				}
				memcpy(Y + v * k, res.data(), sizeof(T) * k);
			}
			at += r->get_size();
		}
	}
	return 0;
}

extern "C" {

uint64_t ref_fg_header_size() { return graph_header::get_header_size(); }
uint64_t ref_fg_vsize(uint32_t ne, uint32_t eds) { return ext_mem_undirected_vertex::num_edges2vsize(ne, eds); }
uint64_t ref_fg_data_off(uint32_t ne, uint32_t eds)
{
	return ext_mem_undirected_vertex::get_edge_data_offset(ne, eds);
}

/* Header fields through graph_header's accessors; -1 unless a graph file of
 * the current version. */
int ref_fg_header(const char *adj, uint64_t *nv, uint64_t *ne, int *eds, int *directed)
{
	const graph_header *h = reinterpret_cast<const graph_header *>(adj);
	if (!h->is_graph_file() || !h->is_right_version()) return -1;
	*nv = h->get_num_vertices();
	*ne = h->get_num_edges();
	*eds = h->get_edge_data_size();
	*directed = h->is_directed_graph() ? 1 : 0;
	return 0;
}

/* dtype 0: FP32 operands, 1: FP64; the edge data (if any) is float. */
int ref_fg_spmm(const char *adj, uint64_t len, int transpose, int dtype, const void *X, void *Y, uint64_t k)
{
	if (len < graph_header::get_header_size()) return -1;
	const graph_header *h = reinterpret_cast<const graph_header *>(adj);
	if (!h->is_graph_file() || !h->is_right_version()) return -1;
	if (h->has_edge_data() && h->get_edge_data_size() != sizeof(float)) return -1;
	if (dtype == 0)
		return walk<float, float>(adj, len, transpose, static_cast<const float *>(X), static_cast<float *>(Y), k);
	return walk<double, float>(adj, len, transpose, static_cast<const double *>(X), static_cast<double *>(Y), k);
}

}
