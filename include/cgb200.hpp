// C++ adapter with the surface of the reference's SINGLE_GPU engine,
// GraphDeviceWorklist (my_project/CGgraph/GraphDevice.cuh:9-269), so that a
// main_partition()-style driver (my_project/CGgraph/main_partition.hpp:319-383)
// swaps engines by changing one type name.  Header-only over the C ABI of
// cgb200.h; link with -lcgb200.
//
//   GraphB200 engine(csrResult, Algorithm_type::BFS);          // uploads the CSR
//   double ms = engine.graphProcess_device(algorithm, root);  // one run, device ms
//   engine.result_D2H();                                      // fills vertexValue
//
// Where the reference calls assert_msg / exit(1), this adapter throws
// cgb200::error carrying the C status code.  vertexValue is uint32[V] for
// BFS / SSSP / CC; after PageRank, vertexValuePr holds double[V] (the
// reference's uint32 PageRank cannot represent the result).
#ifndef CGB200_HPP
#define CGB200_HPP

#include <cstdint>
#include <stdexcept>
#include <string>
#include <vector>

#include "cgb200.h"

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
    std::vector<uint32_t> vertexValue;
    std::vector<double> vertexValuePr;

    GraphB200(const CsrResult& csr, int algorithm, int device = 0, const cgb_options* opt = nullptr)
        : vertexNum(csr.vertexNum), edgeNum(csr.edgeNum), noZeroOutDegreeNum(csr.noZeroOutDegreeNum),
          algorithm_(algorithm), opt_(opt ? *opt : cgb_options{})
    {
        check(cgb_graph_create(csr.csr_offset, csr.csr_dest, csr.csr_weight, csr.vertexNum, csr.edgeNum,
                               csr.noZeroOutDegreeNum, device, &g_));
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
            vertexValuePr.resize(vertexNum);
            check(cgb_graph_result_download(g_, vertexValuePr.data()));
        } else {
            vertexValue.resize(vertexNum);
            check(cgb_graph_result_download(g_, vertexValue.data()));
        }
    }

    // Attaches or replaces the edge weights (cgb_graph_set_weights).
    void setWeights(const uint32_t* weight) { check(cgb_graph_set_weights(g_, weight)); }

    cgb_graph* handle() const { return g_; }

private:
    cgb_graph* g_ = nullptr;
    int algorithm_;
    int last_ = -1;
    cgb_options opt_;
};

}  // namespace cgb200

#endif  // CGB200_HPP
