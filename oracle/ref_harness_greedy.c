/*
 * ref_harness_greedy.c -- test infrastructure, not part of the engine.
 *
 * Compiles the reference's own src/greedy-feature-match.c in place (its main()
 * renamed) and exposes its loader, compute_vertex_features (:527-566),
 * compute_feature_distance (:575-586) and match_vertices (:588-676) to the
 * tests.  Built into oracle/_ref/ by oracle/Makefile.
 */
#define main brain_match_reference_main
#include REF_SRC
#undef main

void* refgreedy_load(const char* path, int* n) { return load_graph(path, n); }
void refgreedy_free(void* g) { free_graph((Graph*)g); }
int refgreedy_node_id(void* g, int idx) { return ((Graph*)g)->node_ids[idx]; }
/* out[6 i + k]: in, out, reachable_2hop, can_reach_2hop, total, original_index,
 * i in the graph's index order (ids ascending) */
void refgreedy_features(void* g, int* out) {
    Graph* G = (Graph*)g;
    VertexFeatures* f = malloc(sizeof(VertexFeatures) * (size_t)G->num_nodes);
    compute_vertex_features(G, f);
    for (int i = 0; i < G->num_nodes; i++) {
        out[6 * i + 0] = f[i].in_degree; out[6 * i + 1] = f[i].out_degree;
        out[6 * i + 2] = f[i].reachable_2hop; out[6 * i + 3] = f[i].can_reach_2hop;
        out[6 * i + 4] = f[i].total_score; out[6 * i + 5] = f[i].original_index;
    }
    free(f);
}
int refgreedy_distance(const int* a, const int* b) {
    VertexFeatures x = {a[0], a[1], a[2], a[3], a[0] + a[1] + a[2] + a[3], 0};
    VertexFeatures y = {b[0], b[1], b[2], b[3], b[0] + b[1] + b[2] + b[3], 0};
    return compute_feature_distance(&x, &y);
}
/* matching[i] = G2 node id matched to G1 vertex index i */
int refgreedy_match(void* g1, void* g2, int* matching) {
    return match_vertices((Graph*)g1, (Graph*)g2, matching);
}
