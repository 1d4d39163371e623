// Oracle harness (test infrastructure only): drives the reference's own
// MULTI_CORE CPU engine, Graph_Numa (my_project/CGgraph/GraphNuma.cuh:9-698),
// on a CSR given as the three raw little-endian files the reference loads
// with load_binFile (Basic/Other/IO.hpp:44-92).  It is compiled by
// oracle/build_ref.sh from the reference sources and is only ever used to
// check and to time the new engine, never as part of it.
//
// usage: cgref_oracle <alg> <V> <E> <offsets.bin> <dest.bin> <weight.bin|-> \
//                     <root[,root...]> <out.bin|-> [runs] [threads]
//   alg: 0 = BFS, 1 = SSSP, 2 = CC  (Algorithm_type, Basic/Graph/basic_struct.hpp:144-151)
//   run i uses root i mod (number of roots).
// Prints one line of JSON: {"alg":..,"runs":..,"ms":[..],"edges":[..],"threads":..},
// where ms is the reference's own graphProcess time of each run and edges
// the run's traversed-edge count (sum of out-degrees of reached vertices).
// The values of the last run (uint32 per vertex, 999999999 = unreachable)
// are written to out.bin.
//
// usage: cgref_oracle reorder <method> <V> <E> <offsets.bin> <dest.bin> <weight.bin|->
//   runs the reference's Reorder::generateReorderGraphFile
//   (my_project/CGgraph/Reorder.hpp:58-241) in its toy-graph mode, which
//   prints the order as a line "old: <old id of new 0> <old id of new 1> ..."
//   and writes no files; the relabelled CSR it builds (get_CSR_reorder) is
//   then printed as "csr_offset:", "csr_dest:" and "csr_weight:" lines.
//
// usage: cgref_oracle edges <V> <edges.bin>
//   runs the reference's edge-list reader on a file of packed 12-byte
//   (src, dst, weight) records: GraphBinReader::group_load_directedGraph,
//   sort_nbr and getStruct_csrResult (Basic/Graph/graphBinReader.hpp:89-325,
//   as main_partition.hpp:105-112 calls them) with one OpenMP thread, since
//   the reader appends to per-vertex vectors from its parallel loop; prints
//   the CSR as above.  Self-loops and duplicates end the process with the
//   reader's own assertions.
//
// usage: cgref_oracle sortnbr <V> <E> <offsets.bin> <dest.bin> <weight.bin>
//   runs nbrSort_taskSteal (my_project/CGgraph/sortNbr.hpp:8-99), the sort the
//   reference driver applies to every loaded CSR (main_partition.hpp:146), and
//   prints the CSR as above; a list with a repeated destination fails its
//   strictly-ascending assert_msg (exit status 1).

#include "Basic/basic_include.cuh"
#include "my_project/CGgraph/host_algorithm.hpp"

// The reference names these PageRank symbols in Graph_Numa::graphProcess
// (my_project/CGgraph/GraphNuma.cuh:222,240,259) but defines them nowhere;
// the harness never runs PageRank through Graph_Numa.
double alpha = 0.85;
double beta = 0.15;
unsigned iteN = 20;
namespace PR_SPACE {
template <typename G>
count_type pr_numa(G&, vertex_id_type, countl_type, countl_type, count_type, bool) { return 0; }
}  // namespace PR_SPACE

#include "my_project/CGgraph/sortNbr.hpp"
#include "my_project/CGgraph/GraphNuma.cuh"
#include "my_project/CGgraph/Reorder.hpp"
#include "Basic/Graph/graphBinReader.hpp"

#include <cstdio>
#include <cstdlib>
#include <string>
#include <unistd.h>
#include <vector>

static void print_u32_line(const char* name, const uint32_t* a, uint64_t n)
{
    printf("\n%s", name);
    for (uint64_t i = 0; i < n; i++) printf(" %u", a[i]);
    printf("\n");
}

static int run_reorder(int argc, char** argv)
{
    if (argc < 8) {
        fprintf(stderr, "usage: %s reorder method V E off dest weight\n", argv[0]);
        return 2;
    }
    int method = atoi(argv[2]);
    uint64_t V = strtoull(argv[3], nullptr, 10);
    uint64_t E = strtoull(argv[4], nullptr, 10);
    if (V == 0) return 2;
    CSR_Result_type csr;
    csr.vertexNum = (count_type)V;
    csr.edgeNum = (countl_type)E;
    csr.csr_offset = load_binFile<countl_type>(argv[5], V + 1);
    csr.csr_dest = E ? load_binFile<vertex_id_type>(argv[6], E) : new vertex_id_type[1];
    if (std::string(argv[7]) != "-" && E) {
        csr.csr_weight = load_binFile<edge_data_type>(argv[7], E);
    } else {
        csr.csr_weight = new edge_data_type[E ? E : 1];
        for (uint64_t i = 0; i < E; i++) csr.csr_weight[i] = 1;
    }
    std::vector<offset_type> outDeg(V), inDeg(V, 0);
    for (uint64_t v = 0; v < V; v++) outDeg[v] = csr.csr_offset[v + 1] - csr.csr_offset[v];
    for (uint64_t e = 0; e < E; e++) inDeg[csr.csr_dest[e]]++;
    Reorder reorder(csr, outDeg.data(), inDeg.data());
    reorder.generateReorderGraphFile((OrderMethod)method, "harness", true);
    CSR_Result_type r = reorder.get_CSR_reorder();
    print_u32_line("csr_offset:", r.csr_offset, V + 1);
    print_u32_line("csr_dest:", r.csr_dest, E);
    print_u32_line("csr_weight:", r.csr_weight, E);
    fflush(stdout);
    _exit(0);
}

static int run_edges(int argc, char** argv)
{
    if (argc < 4) {
        fprintf(stderr, "usage: %s edges V edges.bin\n", argv[0]);
        return 2;
    }
    uint64_t V = strtoull(argv[2], nullptr, 10);
    if (V == 0) return 2;
    reSetThreadNum(1);
    SharedMemory::GraphBinReader reader(GraphRepresentation::CSR);
    reader.group_load_directedGraph(argv[3], (count_type)V);
    reader.sort_nbr();
    CSR_Result_type r;
    reader.getStruct_csrResult(r);
    print_u32_line("csr_offset:", r.csr_offset, V + 1);
    print_u32_line("csr_dest:", r.csr_dest, r.edgeNum);
    print_u32_line("csr_weight:", r.csr_weight, r.edgeNum);
    fflush(stdout);
    _exit(0);
}

static int run_sortnbr(int argc, char** argv)
{
    if (argc < 7) {
        fprintf(stderr, "usage: %s sortnbr V E off dest weight\n", argv[0]);
        return 2;
    }
    uint64_t V = strtoull(argv[2], nullptr, 10);
    uint64_t E = strtoull(argv[3], nullptr, 10);
    if (V == 0) return 2;
    CSR_Result_type csr;
    csr.vertexNum = (count_type)V;
    csr.edgeNum = (countl_type)E;
    csr.csr_offset = load_binFile<countl_type>(argv[4], V + 1);
    csr.csr_dest = E ? load_binFile<vertex_id_type>(argv[5], E) : new vertex_id_type[1];
    csr.csr_weight = E ? load_binFile<edge_data_type>(argv[6], E) : new edge_data_type[1];
    nbrSort_taskSteal(csr);
    print_u32_line("csr_offset:", csr.csr_offset, V + 1);
    print_u32_line("csr_dest:", csr.csr_dest, E);
    print_u32_line("csr_weight:", csr.csr_weight, E);
    fflush(stdout);
    _exit(0);
}

int main(int argc, char** argv)
{
    if (argc > 1 && std::string(argv[1]) == "sortnbr") return run_sortnbr(argc, argv);
    if (argc > 1 && std::string(argv[1]) == "reorder") return run_reorder(argc, argv);
    if (argc > 1 && std::string(argv[1]) == "edges") return run_edges(argc, argv);
    if (argc < 9) {
        fprintf(stderr, "usage: %s alg V E off dest weight root out [runs] [threads]\n", argv[0]);
        return 2;
    }
    int alg = atoi(argv[1]);
    uint64_t V = strtoull(argv[2], nullptr, 10);
    uint64_t E = strtoull(argv[3], nullptr, 10);
    std::string offPath = argv[4], dstPath = argv[5], wPath = argv[6];
    std::vector<uint32_t> roots;
    for (char* p = argv[7]; *p;) {
        roots.push_back((uint32_t)strtoul(p, &p, 10));
        if (*p == ',') p++;
        else if (*p) { fprintf(stderr, "bad root list\n"); return 2; }
    }
    std::string outPath = argv[8];
    int runs = argc > 9 ? atoi(argv[9]) : 1;
    int threads = argc > 10 ? atoi(argv[10]) : 0;
    if (threads > 0) reSetThreadNum(threads);
    bool bad_root = roots.empty();
    for (uint32_t r : roots) bad_root |= r >= V;
    if (alg < 0 || alg > 2 || runs < 1 || V == 0 || bad_root) {
        fprintf(stderr, "bad arguments\n");
        return 2;
    }

    CSR_Result_type csr;
    csr.vertexNum = (count_type)V;
    csr.edgeNum = (countl_type)E;
    csr.csr_offset = load_binFile<countl_type>(offPath, V + 1);
    csr.csr_dest = E ? load_binFile<vertex_id_type>(dstPath, E) : new vertex_id_type[1];
    if (wPath != "-" && E) {
        csr.csr_weight = load_binFile<edge_data_type>(wPath, E);
    } else {
        csr.csr_weight = new edge_data_type[E ? E : 1];
        for (uint64_t i = 0; i < E; i++) csr.csr_weight[i] = 1;
    }
    csr.noZeroOutDegreeNum = (count_type)V;

    // The reference driver sorts every neighbour list and asserts strictly
    // ascending destinations before any engine runs (main_partition.hpp:146).
    nbrSort_taskSteal(csr);

    // Graph_Numa frees the arrays it is given (GraphNuma.cuh:417-419).
    Graph_Numa* engine = new Graph_Numa(csr);
    std::string ms = "[", edges = "[";
    for (int r = 0; r < runs; r++) {
        double t = engine->graphProcess((Algorithm_type)alg, roots[r % roots.size()]);
        unsigned long long m = 0;
        for (uint64_t v = 0; v < V; v++)
            if (engine->vertexValue[v] != VertexValue_MAX) m += engine->outDegree[v];
        char buf[96];
        snprintf(buf, sizeof(buf), "%s%.6f", r ? "," : "", t);
        ms += buf;
        snprintf(buf, sizeof(buf), "%s%llu", r ? "," : "", m);
        edges += buf;
    }
    ms += "]";
    edges += "]";

    if (outPath != "-") {
        FILE* f = fopen(outPath.c_str(), "wb");
        if (!f) { fprintf(stderr, "cannot open %s\n", outPath.c_str()); _exit(3); }
        size_t n = fwrite(engine->vertexValue, sizeof(vertex_data_type), V, f);
        fclose(f);
        if (n != V) _exit(3);
    }
    printf("\n{\"alg\": %d, \"runs\": %d, \"ms\": %s, \"edges\": %s, \"threads\": %llu}\n", alg, runs,
           ms.c_str(), edges.c_str(), (unsigned long long)ThreadNum);
    fflush(stdout);
    // DoubleBuffer<dense_bitset> frees the frontier bitmaps twice when the
    // engine is destroyed; leave without running destructors.
    _exit(0);
}
