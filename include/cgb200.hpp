// C++ adapter with the surface of the reference's SINGLE_GPU engine,
// GraphDeviceWorklist (my_project/CGgraph/GraphDevice.cuh:9-269), so that a
// main_partition()-style driver (my_project/CGgraph/main_partition.hpp:319-383)
// swaps engines by changing one type name (and reads PageRank results from
// vertexValuePr).  Header-only over the C ABI of
// cgb200.h; link with -lcgb200.
//
//   GraphB200 engine(csrResult, Algorithm_type::BFS);          // uploads the CSR
//   double ms = engine.graphProcess_device(algorithm, root);  // one run, device ms
//   engine.result_D2H();                                      // fills vertexValue
//
// Where the reference calls assert_msg / exit(1), this adapter throws
// cgb200::error carrying the C status code.  vertexValue is a raw pointer to
// uint32[V] host values for BFS / SSSP / CC, owned by the engine as the
// reference's is (GraphDevice.cuh:21,183); after PageRank, vertexValuePr
// points at double[V] (the reference's uint32 PageRank cannot represent the
// result).
#ifndef CGB200_HPP
#define CGB200_HPP

#include <cstdint>
#include <cstdio>
#include <stdexcept>
#include <string>
#include <vector>

#include "cgb200.h"
#include "cgb200_gen.h"

namespace cgb200 {

class error : public std::runtime_error {
public:
    error(cgb_status s, const std::string& what) : std::runtime_error(what), status(s) {}
    cgb_status status;
};

inline void check(cgb_status s)
{
    if (s != CGB_OK) throw error(s, std::string(cgb_status_string(s)) + ": " + cgb_last_error_string());
}

// Any struct with the members of CSR_Result_type (Basic/Graph/basic_struct.hpp:7-16).
template <typename CsrResult>
class GraphB200 {
public:
    uint32_t vertexNum = 0;
    uint32_t edgeNum = 0;
    uint32_t noZeroOutDegreeNum = 0;
    uint32_t* vertexValue = nullptr;  // uint32[V], valid for the engine's lifetime
    double* vertexValuePr = nullptr;  // double[V], valid for the engine's lifetime

    GraphB200(const CsrResult& csr, int algorithm, int device = 0, const cgb_options* opt = nullptr)
        : vertexNum(csr.vertexNum), edgeNum(csr.edgeNum), noZeroOutDegreeNum(csr.noZeroOutDegreeNum),
          algorithm_(algorithm), opt_(opt ? *opt : cgb_options{})
    {
        check(cgb_graph_create(csr.csr_offset, csr.csr_dest, csr.csr_weight, csr.vertexNum, csr.edgeNum,
                               csr.noZeroOutDegreeNum, device, &g_));
        allocValues();
    }
    // The reference's other input (has_csrFile = 0, main_partition.hpp:105-116):
    // a binary edge list of 12-byte (src, dst, weight) records, built into the
    // CSR on the device (cgb_graph_load_edge_file).
    GraphB200(const std::string& edge_file, uint32_t vertices, int algorithm, int device = 0,
              const cgb_options* opt = nullptr)
        : algorithm_(algorithm), opt_(opt ? *opt : cgb_options{})
    {
        check(cgb_graph_load_edge_file(edge_file.c_str(), vertices, device, &g_));
        check(cgb_graph_info(g_, &vertexNum, &edgeNum, nullptr));
        noZeroOutDegreeNum = vertexNum;
        allocValues();
    }
    GraphB200(const GraphB200&) = delete;
    GraphB200& operator=(const GraphB200&) = delete;
    ~GraphB200() { cgb_graph_destroy(g_); }

    // GraphDevice.cuh:92-176.  For PageRank `root` is the iteration count.
    double graphProcess_device(int algorithm, uint32_t root = 0)
    {
        double ms = 0;
        check(cgb_run(g_, algorithm, root, &opt_, nullptr, nullptr, &ms));
        last_ = algorithm;
        return ms;
    }

    // GraphDevice.cuh:259-262.
    void result_D2H()
    {
        if (last_ == CGB_PR) {
            pr_.resize(vertexNum);
            vertexValuePr = pr_.data();
            check(cgb_graph_result_download(g_, vertexValuePr));
        } else {
            check(cgb_graph_result_download(g_, vertexValue));
        }
    }

    // Attaches or replaces the edge weights (cgb_graph_set_weights).
    void setWeights(const uint32_t* weight) { check(cgb_graph_set_weights(g_, weight)); }

    cgb_graph* handle() const { return g_; }

private:
    void allocValues()
    {
        values_.assign(vertexNum, 0u);
        vertexValue = values_.data();
    }

    cgb_graph* g_ = nullptr;
    int algorithm_;
    int last_ = -1;
    cgb_options opt_;
    std::vector<uint32_t> values_;
    std::vector<double> pr_;
};

// The surface of the reference's Reorder (my_project/CGgraph/Reorder.hpp:6-60,
// 243-246, 538-620) over cgb_graph_reorder: the order and the relabelled CSR
// are built on the device, so the degree arrays the reference's constructor
// takes are not needed.  generateReorderGraphFile writes the five files of
// saveCSR_reorderFile (offsets, dest, weight, old2new, addition = the number
// of vertices without out-edges, absent for IN_DEGREE_DEC); the reference
// derives their names from its graph folder, here they are given.  The
// relabelled lists are sorted by new id, as the reference's driver sorts them
// after loading (main_partition.hpp:146).
//
//   cgb200::ReorderB200<CSR_Result_type> reorder(csrResult);
//   reorder.generateReorderGraphFile(CGB_ORDER_MY_BFS_OUT, off, dest, weight, old2new, addition);
//   CSR_Result_type r = reorder.get_CSR_reorder();   // host arrays owned by `reorder`
template <typename CsrResult>
class ReorderB200 {
public:
    uint32_t vertexNum = 0;
    uint32_t edgeNum = 0;
    uint32_t zeroOutDegreeNum = 0;
    std::vector<uint32_t> old2new;

    explicit ReorderB200(const CsrResult& csr, int device = 0) : vertexNum(csr.vertexNum), edgeNum(csr.edgeNum)
    {
        check(cgb_graph_create(csr.csr_offset, csr.csr_dest, csr.csr_weight, csr.vertexNum, csr.edgeNum,
                               csr.vertexNum, device, &g_));
    }
    ReorderB200(const ReorderB200&) = delete;
    ReorderB200& operator=(const ReorderB200&) = delete;
    ~ReorderB200() { cgb_graph_destroy(g_); }

    // Builds the order and the relabelled CSR (host copies kept for
    // get_CSR_reorder); writes the files when their names are non-empty.
    void generateReorderGraphFile(int orderMethod, const std::string& csrOffsetFile = "",
                                  const std::string& csrDestFile = "", const std::string& csrWeightFile = "",
                                  const std::string& old2newFile = "", const std::string& additionFile = "")
    {
        cgb_graph* r = nullptr;
        uint32_t nz = 0;
        old2new.resize(vertexNum);
        check(cgb_graph_reorder(g_, orderMethod, old2new.data(), &nz, &r));
        off_.resize((size_t)vertexNum + 1);
        dst_.resize(edgeNum ? edgeNum : 1);
        w_.resize(edgeNum ? edgeNum : 1);
        const cgb_status st = cgb_graph_download(r, off_.data(), dst_.data(), w_.data());
        cgb_graph_destroy(r);
        check(st);
        zeroOutDegreeNum = vertexNum - nz;
        write(csrOffsetFile, off_.data(), (size_t)vertexNum + 1);
        write(csrDestFile, dst_.data(), edgeNum);
        write(csrWeightFile, w_.data(), edgeNum);
        write(old2newFile, old2new.data(), vertexNum);
        if (orderMethod == CGB_ORDER_IN_DEGREE_DEC) write(additionFile, nullptr, 0);
        else write(additionFile, &zeroOutDegreeNum, 1);
    }

    CsrResult get_CSR_reorder()
    {
        CsrResult c{};
        c.vertexNum = vertexNum;
        c.edgeNum = edgeNum;
        c.csr_offset = off_.data();
        c.csr_dest = dst_.data();
        c.csr_weight = w_.data();
        c.noZeroOutDegreeNum = vertexNum - zeroOutDegreeNum;
        return c;
    }

private:
    static void write(const std::string& path, const uint32_t* a, size_t n)
    {
        if (path.empty()) return;
        FILE* f = std::fopen(path.c_str(), "wb");
        if (!f) throw error(CGB_EIO, "cannot open " + path);
        const size_t m = n ? std::fwrite(a, sizeof(uint32_t), n, f) : 0;
        const bool ok = std::fclose(f) == 0 && m == n;
        if (!ok) throw error(CGB_EIO, "cannot write " + path);
    }

    cgb_graph* g_ = nullptr;
    std::vector<uint32_t> off_, dst_, w_;
};

}  // namespace cgb200

#endif  // CGB200_HPP
