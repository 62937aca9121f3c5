// comm.h -- the ranks of a multi-process run: the Cartesian rank layout of
// comm/comm.impala:221-299 (get_node_config, get_node_bounding_box) with the
// periodic MPI cart of comm/mpi.cpp:19-49, and the transport that carries the
// halo and migration messages between ranks.
//
// One process per GPU.  The world size and rank come from the environment
// (TINYMD_WORLD_SIZE / TINYMD_RANK, else WORLD_SIZE / RANK as torchrun sets them,
// else OMPI_COMM_WORLD_SIZE / OMPI_COMM_WORLD_RANK, else PMI_SIZE / PMI_RANK);
// md_mpi_initialize connects the ranks.  Control traffic (counts, reductions,
// barriers) always goes over a TCP mesh; bulk data goes GPU to GPU through NCCL
// when every rank has its own device, else through page-locked host buffers
// over the same mesh (ranks that share a device).
#pragma once

#include <cuda_runtime.h>

#include <string>
#include <vector>

namespace tmd {

// Neighbour regions of a rank box: type t = ez*9 + ey*3 + ex - 1 (e per axis: 0 inside,
// 1 beyond the upper face, 2 beyond the lower face), the ghost-type numbering of the
// border pass.
struct Topology {
    int world = 1, rank = 0;
    int dims[3] = {1, 1, 1};
    int coords[3] = {0, 0, 0};
    int peer[26];        // rank owning region t
    int shift[26][3];    // world lengths added to a position sent into region t
    unsigned selfmask;   // bit t: region t is this rank itself (a periodic image of its own atoms)
    std::vector<int> peers;  // the distinct other ranks among peer[], ascending
};

// comm/comm.impala:221-257 (the loops run i, j over [1, n), as the reference's range does)
void node_config(int world, const double len[3], int dims[3]);
// the periodic row-major cart of comm/mpi.cpp:19-49 and the 26 regions around `rank`
void make_topology(int world, int rank, const int dims[3], Topology& t);
// comm/comm.impala:260-299
void rank_box(const double world_aabb[6], const int dims[3], const int coords[3], double box[6]);

struct HostMsg {
    int peer;
    void* data;
    size_t bytes;
};

class Comm {
public:
    int world() const { return world_; }
    int rank() const { return rank_; }
    bool active() const { return world_ > 1; }
    bool device_direct() const { return nccl_ != nullptr; }
    const char* transport() const { return nccl_ ? "nccl" : (world_ > 1 ? "socket" : "none"); }
    const std::string& error() const { return err_; }

    // reads the environment; world 1 needs nothing else.  Returns false (error() says why)
    // when the ranks cannot be connected.
    bool init();
    void finalize();

    // every listed message sent and received (at most one of each per peer); blocks
    bool exchange(const std::vector<HostMsg>& sends, const std::vector<HostMsg>& recvs);
    // device buffers, enqueued on `stream` (NCCL only)
    bool exchange_device(const std::vector<HostMsg>& sends, const std::vector<HostMsg>& recvs, cudaStream_t stream);
    // reductions in rank order (the same result on every rank)
    bool allreduce_sum(double* v, int n);
    bool allreduce_max(double* v, int n);
    bool allreduce_sum(long long* v, int n);
    bool barrier();

    Topology topo;
    bool topo_set = false;

private:
    template <class T, class Op>
    bool allreduce(T* v, int n, Op op);
    bool fail(const std::string& why);

    int world_ = 1, rank_ = 0;
    std::vector<int> fd_;  // mesh socket per peer rank (-1 for self)
    void* nccl_ = nullptr;  // ncclComm_t
    std::string err_;
};

Comm& comm();

}  // namespace tmd
