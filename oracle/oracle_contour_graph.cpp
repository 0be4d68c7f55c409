// Test infrastructure: the contour-construction test graphs of the reference and its CPU
// reference (UnitTest/test_parallel_contour_construction.cpp), restated.
//
// A graph is undirected with a 0/1 "flip" weight per edge, stored as CSR with both directions
// of every edge (make_undirected_csr, 28-56). The eight cases of the test's main (609-668) are
// built in its order from one std::mt19937(42): a fixed 14-node graph, chains (some closed into
// cycles), grids, random sparse components (random spanning tree + extra edges) and singletons
// with pairs. The CPU reference (cpu_reference, 144-187) is a breadth-first flood from the
// smallest unvisited node with parity 0 at the seed, a node's parity the seed's XOR the flips
// along its discovery path, and an "inconsistent" flag for any edge whose endpoints' parities
// disagree with its flip.
//
// The generators draw from libstdc++'s uniform_int_distribution and shuffle; the graphs equal
// the test's where its standard library draws the same. The test holds no stored outputs: it
// checks a second implementation against the flood, which is what this file serves.
#include <algorithm>
#include <cstdint>
#include <deque>
#include <numeric>
#include <random>
#include <tuple>
#include <vector>

namespace
{
	using uint = uint32_t;
	using Edge = std::tuple<uint, uint, uint>; // (u, v, flip)

	struct CsrGraph
	{
		uint n = 0;
		std::vector<uint> row_ptr, col, flip;
	};

	CsrGraph to_csr(uint n, const std::vector<Edge>& edges)
	{
		CsrGraph g;
		g.n = n;
		g.row_ptr.assign(n + 1, 0u);
		for (const auto& [u, v, w] : edges)
		{
			g.row_ptr[u + 1]++;
			g.row_ptr[v + 1]++;
		}
		std::partial_sum(g.row_ptr.begin(), g.row_ptr.end(), g.row_ptr.begin());
		g.col.resize(g.row_ptr[n]);
		g.flip.resize(g.row_ptr[n]);
		std::vector<uint> at(g.row_ptr.begin(), g.row_ptr.end() - 1);
		for (const auto& [u, v, w] : edges)
		{
			const uint a = at[u]++, b = at[v]++;
			g.col[a] = v;
			g.flip[a] = w & 1u;
			g.col[b] = u;
			g.flip[b] = w & 1u;
		}
		return g;
	}

	// num_chains chains of chain_length nodes; the first num_cycles closed into cycles
	CsrGraph chains(uint num_chains, uint chain_length, uint num_cycles, std::mt19937& rng)
	{
		std::uniform_int_distribution<uint> flip(0, 1);
		std::vector<Edge> edges;
		for (uint c = 0; c < num_chains; c++)
		{
			const uint b = c * chain_length;
			for (uint i = 0; i + 1 < chain_length; i++)
				edges.emplace_back(b + i, b + i + 1, flip(rng));
			if (c < num_cycles && chain_length >= 3)
				edges.emplace_back(b, b + chain_length - 1, flip(rng));
		}
		return to_csr(num_chains * chain_length, edges);
	}

	// rows x cols grid, right then down neighbour of each node in row-major order
	CsrGraph grid(uint rows, uint cols, std::mt19937& rng)
	{
		std::uniform_int_distribution<uint> flip(0, 1);
		std::vector<Edge> edges;
		for (uint r = 0; r < rows; r++)
			for (uint c = 0; c < cols; c++)
			{
				const uint i = r * cols + c;
				if (c + 1 < cols)
					edges.emplace_back(i, i + 1, flip(rng));
				if (r + 1 < rows)
					edges.emplace_back(i, i + cols, flip(rng));
			}
		return to_csr(rows * cols, edges);
	}

	// n nodes in num_components consecutive groups (the last takes the remainder), each a
	// shuffled path (a random spanning tree) plus extra random edges up to avg_degree
	CsrGraph random_sparse(uint n, uint avg_degree, uint num_components, std::mt19937& rng)
	{
		std::uniform_int_distribution<uint> flip(0, 1);
		std::vector<Edge> edges;
		const uint size = std::max(n / std::max(num_components, 1u), 1u);
		for (uint c = 0; c < num_components; c++)
		{
			const uint lo = c * size, hi = c + 1 == num_components ? n : lo + size;
			const uint sz = hi - lo;
			if (sz <= 1)
				continue;
			std::vector<uint> order(sz);
			std::iota(order.begin(), order.end(), lo);
			std::shuffle(order.begin(), order.end(), rng);
			for (uint i = 0; i + 1 < sz; i++)
				edges.emplace_back(std::min(order[i], order[i + 1]), std::max(order[i], order[i + 1]), flip(rng));
			const int extra = std::max(int(sz * avg_degree / 2) - int(sz - 1), 0);
			std::uniform_int_distribution<uint> node(lo, hi - 1);
			for (int i = 0; i < extra; i++)
			{
				const uint u = node(rng);
				const uint v = node(rng);
				if (u != v)
					edges.emplace_back(std::min(u, v), std::max(u, v), flip(rng));
			}
		}
		return to_csr(n, edges);
	}

	// case `which` (0-7) of the test's sequence; the cases before it are drawn first, as the
	// test shares one generator across them
	CsrGraph test_case(int which)
	{
		std::mt19937 rng(42);
		CsrGraph g;
		for (int k = 0; k <= which; k++)
		{
			switch (k)
			{
			case 0: // fixed: a chain, a consistent 3-cycle, a singleton (6), a chain, an inconsistent triangle
				g = to_csr(14, { { 0, 1, 1 }, { 1, 2, 0 }, { 3, 4, 1 }, { 4, 5, 1 }, { 5, 3, 0 }, { 7, 8, 0 }, { 8, 9, 1 }, { 9, 10, 1 },
								   { 11, 12, 1 }, { 12, 13, 1 }, { 13, 11, 1 } });
				break;
			case 1:
				g = chains(10000, 10, 500, rng);
				break;
			case 2:
				g = chains(1000, 100, 200, rng);
				break;
			case 3:
				g = grid(100, 100, rng);
				break;
			case 4:
				g = grid(200, 250, rng);
				break;
			case 5:
				g = random_sparse(50000, 4, 100, rng);
				break;
			case 6:
				g = random_sparse(100000, 6, 500, rng);
				break;
			default:
			{
				// 50,000 singletons, then 25,000 pairs
				std::uniform_int_distribution<uint> flip(0, 1);
				std::vector<Edge> edges;
				for (uint i = 50000; i < 100000; i += 2)
					edges.emplace_back(i, i + 1, flip(rng));
				g = to_csr(100000, edges);
			}
			}
		}
		return g;
	}
} // namespace

extern "C"
{
	void* oracle_cc_graph_make(int which)
	{
		if (which < 0 || which > 7)
			return nullptr;
		return new CsrGraph(test_case(which));
	}
	void oracle_cc_graph_size(const void* h, uint* n, uint* m)
	{
		const CsrGraph* g = static_cast<const CsrGraph*>(h);
		*n = g->n;
		*m = uint(g->col.size());
	}
	void oracle_cc_graph_copy(const void* h, uint* row_ptr, uint* col, uint* flip)
	{
		const CsrGraph* g = static_cast<const CsrGraph*>(h);
		std::copy(g->row_ptr.begin(), g->row_ptr.end(), row_ptr);
		std::copy(g->col.begin(), g->col.end(), col);
		std::copy(g->flip.begin(), g->flip.end(), flip);
	}
	void oracle_cc_graph_free(void* h) { delete static_cast<CsrGraph*>(h); }

	// the test's CPU reference: root[i] = the seed (smallest node) of i's component,
	// parity[i]; returns 1 when some edge's endpoints disagree with its flip
	uint oracle_cc_bfs(uint n, const uint* row_ptr, const uint* col, const uint* flip, uint* root, uint* parity)
	{
		std::vector<uint8_t> seen(n, 0);
		bool bad = false;
		for (uint s = 0; s < n; s++)
		{
			if (seen[s])
				continue;
			seen[s] = 1;
			root[s] = s;
			parity[s] = 0;
			std::deque<uint> q{ s };
			while (!q.empty())
			{
				const uint u = q.front();
				q.pop_front();
				for (uint e = row_ptr[u]; e < row_ptr[u + 1]; e++)
				{
					const uint v = col[e], want = parity[u] ^ (flip[e] & 1u);
					if (!seen[v])
					{
						seen[v] = 1;
						root[v] = s;
						parity[v] = want;
						q.push_back(v);
					}
					else if (parity[v] != want)
						bad = true;
				}
			}
		}
		return bad ? 1u : 0u;
	}
}
