// Regenerates the random edge list of FlashX's matrix/unit-test/
// test-sparse_matrix.cpp:40-72 (create_rand_el): 100,000 draws of
// (random() % 16384, random() % 16384) from glibc's default-seeded random(),
// deduplicated by an unordered_set whose hash is first + second, listed in
// that set's iteration order with value = position (as float).  Prints
// "src dst" per line.  Fixture generator only (tests/golden/make_golden.py).
#include <cstdio>
#include <cstdlib>
#include <cstdint>
#include <unordered_set>
#include <utility>

typedef std::pair<uint32_t, uint32_t> edge_t;
struct hash_edge { size_t operator()(const edge_t &e) const { return e.first + e.second; } };
struct edge_equal { bool operator()(const edge_t &a, const edge_t &b) const { return a.first == b.first && a.second == b.second; } };

int main()
{
	const int num_rows = 1024 * 16, num_cols = 1024 * 16;
	std::unordered_set<edge_t, hash_edge, edge_equal> edges;
	for (size_t i = 0; i < 100000; i++) {
		edge_t e;
		e.first = random() % num_rows;
		e.second = random() % num_cols;
		edges.insert(e);
	}
	for (const edge_t &e : edges) printf("%u %u\n", e.first, e.second);
	return 0;
}
