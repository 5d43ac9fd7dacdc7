// Minimal stand-in for the few Boost Graph names that the reference's
// src/testSssp.cpp mentions, so that its own SimpleReferenceSssp (the CPU SSSP check)
// compiles without Boost. Only declarations needed to compile BoostReferenceSssp are
// given; calling dijkstra_shortest_paths here aborts (the oracle never calls ssspBoost).
// Part of the oracle recipe (test infrastructure), never of the product.
#ifndef APSPIE_ORACLE_BOOST_SHIM
#define APSPIE_ORACLE_BOOST_SHIM
#include <cstdio>
#include <cstdlib>
#include <tuple>
#include <utility>

namespace boost {
struct vecS {};
struct directedS {};
struct no_property {};
struct edge_weight_t {};
struct vertex_index_t {};
static const vertex_index_t vertex_index = vertex_index_t();
template <class Tag, class T> struct property {};

struct counting_vertex_iterator {
    int v;
    int operator*() const { return v; }
    counting_vertex_iterator &operator++() { ++v; return *this; }
    bool operator!=(const counting_vertex_iterator &o) const { return v != o.v; }
};

template <class A, class B, class C, class D, class E>
struct adjacency_list {
    int n;
    template <class EIt, class WIt>
    adjacency_list(EIt, EIt, WIt, int nv) : n(nv) {}
};

template <class G> struct graph_traits {
    typedef int vertex_descriptor;
    typedef int edge_descriptor;
    typedef counting_vertex_iterator vertex_iterator;
};

template <class G, class Tag> struct property_map { typedef int type; };

template <class G> int vertex(int i, const G &) { return i; }
template <class G> int get(vertex_index_t, const G &) { return 0; }
template <class It, class IM> It make_iterator_property_map(It it, IM) { return it; }

struct dijkstra_params {
    template <class It> dijkstra_params distance_map(It) const { return *this; }
};
template <class It> dijkstra_params predecessor_map(It) { return dijkstra_params(); }
template <class It> dijkstra_params distance_map(It) { return dijkstra_params(); }
template <class G, class V>
void dijkstra_shortest_paths(const G &, V, const dijkstra_params &) {
    std::fprintf(stderr, "boost shim: dijkstra_shortest_paths is not available\n");
    std::abort();
}
template <class G>
std::pair<counting_vertex_iterator, counting_vertex_iterator> vertices(const G &g) {
    return std::make_pair(counting_vertex_iterator{0}, counting_vertex_iterator{g.n});
}
using std::tie;
}  // namespace boost
#endif
