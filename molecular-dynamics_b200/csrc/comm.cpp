// comm.cpp -- rank layout and transport of a multi-process run (see comm.h).
//
// The reference runs its ranks over MPI (comm/mpi.impala, comm/mpi.cpp) and stages every
// message through host memory.  Here the ranks meet over TCP (rank 0 listens, the others
// connect; then every pair of ranks holds one connection), which carries the counts,
// reductions and barriers.  Halo and migration payloads go device to device through NCCL
// when every rank owns a different GPU (NVLink / NVSwitch on one node), else through
// page-locked host buffers over the TCP mesh.  libnccl is opened at run time, so a
// single-process user never loads it.

#include "comm.h"

#include <arpa/inet.h>
#include <dlfcn.h>
#include <netdb.h>
#include <netinet/in.h>
#include <netinet/tcp.h>
#include <poll.h>
#include <sys/socket.h>
#include <unistd.h>

#include <nccl.h>

#include <algorithm>
#include <cerrno>
#include <chrono>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <type_traits>

namespace tmd {

// ---- rank layout -------------------------------------------------------------------------
void node_config(int world, const double len[3], int dims[3]) {
    const double areax = len[0] * len[1];
    const double areay = len[0] * len[2];
    const double areaz = len[1] * len[2];
    double best = 2.0 * (areax + areay + areaz);
    dims[0] = dims[1] = dims[2] = 1;
    for (int i = 1; i < world; ++i) {
        if (world % i != 0) continue;
        const int rem = world / i;
        for (int j = 1; j < rem; ++j) {
            if (rem % j != 0) continue;
            const int k = rem / j;
            const double surf = areax / i / j + areay / i / k + areaz / j / k;
            if (surf < best) {
                dims[0] = i;
                dims[1] = j;
                dims[2] = k;
                best = surf;
            }
        }
    }
}

void make_topology(int world, int rank, const int dims[3], Topology& t) {
    t.world = world;
    t.rank = rank;
    for (int d = 0; d < 3; ++d) t.dims[d] = dims[d];
    // MPI_Cart_create without reordering: row-major, the last axis fastest
    t.coords[2] = rank % dims[2];
    t.coords[1] = (rank / dims[2]) % dims[1];
    t.coords[0] = rank / (dims[1] * dims[2]);
    t.selfmask = 0;
    t.peers.clear();
    for (int tt = 1; tt < 27; ++tt) {
        const int e[3] = {tt % 3, (tt / 3) % 3, tt / 9};
        int c[3];
        for (int d = 0; d < 3; ++d) {
            c[d] = t.coords[d] + (e[d] == 1 ? 1 : (e[d] == 2 ? -1 : 0));
            int sh = 0;
            // a region past the upper world face is the low end of the periodic box: the image of
            // a position sent there lies one box length lower (and the other way round)
            if (c[d] >= dims[d]) { c[d] -= dims[d]; sh = -1; }
            if (c[d] < 0) { c[d] += dims[d]; sh = 1; }
            t.shift[tt - 1][d] = sh;
        }
        const int p = (c[0] * dims[1] + c[1]) * dims[2] + c[2];
        t.peer[tt - 1] = p;
        if (p == rank) t.selfmask |= 1u << (tt - 1);
        else if (std::find(t.peers.begin(), t.peers.end(), p) == t.peers.end()) t.peers.push_back(p);
    }
    std::sort(t.peers.begin(), t.peers.end());
}

void rank_box(const double w[6], const int dims[3], const int coords[3], double box[6]) {
    for (int d = 0; d < 3; ++d) {
        const double len = (w[2 * d + 1] - w[2 * d]) / (double)dims[d];
        const double lo = w[2 * d] + len * (double)coords[d];
        box[2 * d] = lo;
        box[2 * d + 1] = lo + len;
    }
}

// ---- NCCL, opened at run time ----------------------------------------------------------------
struct Nccl {
    void* so = nullptr;
    ncclResult_t (*get_unique_id)(ncclUniqueId*) = nullptr;
    ncclResult_t (*init_rank)(ncclComm_t*, int, ncclUniqueId, int) = nullptr;
    ncclResult_t (*destroy)(ncclComm_t) = nullptr;
    ncclResult_t (*group_start)() = nullptr;
    ncclResult_t (*group_end)() = nullptr;
    ncclResult_t (*send)(const void*, size_t, ncclDataType_t, int, ncclComm_t, cudaStream_t) = nullptr;
    ncclResult_t (*recv)(void*, size_t, ncclDataType_t, int, ncclComm_t, cudaStream_t) = nullptr;
    const char* (*error_string)(ncclResult_t) = nullptr;

    bool open() {
        if (so) return true;
        so = dlopen("libnccl.so.2", RTLD_NOW | RTLD_LOCAL);
        if (!so) return false;
        bool ok = true;
        auto sym = [&](auto& fn, const char* name) {
            fn = reinterpret_cast<std::remove_reference_t<decltype(fn)>>(dlsym(so, name));
            ok = ok && fn != nullptr;
        };
        sym(get_unique_id, "ncclGetUniqueId");
        sym(init_rank, "ncclCommInitRank");
        sym(destroy, "ncclCommDestroy");
        sym(group_start, "ncclGroupStart");
        sym(group_end, "ncclGroupEnd");
        sym(send, "ncclSend");
        sym(recv, "ncclRecv");
        sym(error_string, "ncclGetErrorString");
        if (!ok) {
            dlclose(so);
            so = nullptr;
        }
        return ok;
    }
};
Nccl g_nccl;

namespace {

// ---- sockets -------------------------------------------------------------------------------------
double now_s() {
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

const char* env_first(std::initializer_list<const char*> names) {
    for (const char* n : names) {
        const char* v = std::getenv(n);
        if (v && *v) return v;
    }
    return nullptr;
}

double timeout_s() {
    const char* v = std::getenv("TINYMD_COMM_TIMEOUT");
    const double t = v ? std::atof(v) : 0.0;
    return t > 0.0 ? t : 300.0;
}

void tune(int fd) {
    int one = 1;
    setsockopt(fd, IPPROTO_TCP, TCP_NODELAY, &one, sizeof(one));
}

// blocking transfer of exactly n bytes, giving up after `limit` seconds without progress
bool io_all(int fd, void* buf, size_t n, bool out, double limit) {
    char* p = static_cast<char*>(buf);
    double last = now_s();
    while (n > 0) {
        pollfd pf{fd, (short)(out ? POLLOUT : POLLIN), 0};
        const int r = poll(&pf, 1, 500);
        if (r < 0 && errno != EINTR) return false;
        if (r <= 0) {
            if (now_s() - last > limit) return false;
            continue;
        }
        const ssize_t k = out ? ::send(fd, p, n, MSG_NOSIGNAL | MSG_DONTWAIT) : ::recv(fd, p, n, MSG_DONTWAIT);
        if (k == 0 && !out) return false;  // peer closed
        if (k < 0) {
            if (errno == EAGAIN || errno == EWOULDBLOCK || errno == EINTR) continue;
            return false;
        }
        p += k;
        n -= (size_t)k;
        last = now_s();
    }
    return true;
}

int listen_on(uint16_t port, uint16_t* bound) {
    const int fd = socket(AF_INET, SOCK_STREAM, 0);
    if (fd < 0) return -1;
    int one = 1;
    setsockopt(fd, SOL_SOCKET, SO_REUSEADDR, &one, sizeof(one));
    sockaddr_in a{};
    a.sin_family = AF_INET;
    a.sin_addr.s_addr = htonl(INADDR_ANY);
    a.sin_port = htons(port);
    if (bind(fd, (sockaddr*)&a, sizeof(a)) != 0 || listen(fd, 256) != 0) {
        close(fd);
        return -1;
    }
    socklen_t len = sizeof(a);
    getsockname(fd, (sockaddr*)&a, &len);
    if (bound) *bound = ntohs(a.sin_port);
    return fd;
}

int accept_one(int lfd, double limit, uint32_t* peer_ip) {
    const double t0 = now_s();
    while (now_s() - t0 < limit) {
        pollfd pf{lfd, POLLIN, 0};
        const int r = poll(&pf, 1, 500);
        if (r < 0 && errno != EINTR) return -1;
        if (r <= 0) continue;
        sockaddr_in a{};
        socklen_t len = sizeof(a);
        const int fd = accept(lfd, (sockaddr*)&a, &len);
        if (fd < 0) continue;
        if (peer_ip) *peer_ip = a.sin_addr.s_addr;
        tune(fd);
        return fd;
    }
    return -1;
}

// connects to ip:port (network order ip), retrying until the listener is up
int connect_to(uint32_t ip, uint16_t port, double limit) {
    const double t0 = now_s();
    while (now_s() - t0 < limit) {
        const int fd = socket(AF_INET, SOCK_STREAM, 0);
        if (fd < 0) return -1;
        sockaddr_in a{};
        a.sin_family = AF_INET;
        a.sin_addr.s_addr = ip;
        a.sin_port = htons(port);
        if (connect(fd, (sockaddr*)&a, sizeof(a)) == 0) {
            tune(fd);
            return fd;
        }
        close(fd);
        usleep(100000);
    }
    return -1;
}

bool resolve(const char* host, uint32_t* ip) {
    addrinfo hints{};
    hints.ai_family = AF_INET;
    hints.ai_socktype = SOCK_STREAM;
    addrinfo* res = nullptr;
    if (getaddrinfo(host, nullptr, &hints, &res) != 0 || !res) return false;
    *ip = ((sockaddr_in*)res->ai_addr)->sin_addr.s_addr;
    freeaddrinfo(res);
    return true;
}

constexpr uint32_t kMagic = 0x746d6431u;  // "tmd1"

struct Hello {
    uint32_t magic;
    int32_t rank, world;
    uint16_t port;
    uint8_t nccl_ok, pad;
    uint8_t uuid[16];
};

struct Entry {
    uint32_t ip;
    uint16_t port;
    uint16_t pad;
};

}  // namespace

// ---- Comm ----------------------------------------------------------------------------------------
Comm& comm() {
    static Comm c;
    return c;
}

bool Comm::fail(const std::string& why) {
    err_ = why;
    return false;
}

bool Comm::init() {
    if (world_ > 1) return true;  // already connected
    err_.clear();
    const char* pairs[4][2] = {{"TINYMD_WORLD_SIZE", "TINYMD_RANK"},
                               {"WORLD_SIZE", "RANK"},
                               {"OMPI_COMM_WORLD_SIZE", "OMPI_COMM_WORLD_RANK"},
                               {"PMI_SIZE", "PMI_RANK"}};
    int w = 1, r = 0;
    for (auto& pr : pairs) {
        const char* ws = std::getenv(pr[0]);
        const char* rs = std::getenv(pr[1]);
        if (ws && rs) {
            w = std::atoi(ws);
            r = std::atoi(rs);
            break;
        }
    }
    if (w <= 1) {
        world_ = 1;
        rank_ = 0;
        return true;
    }
    if (r < 0 || r >= w) return fail("rank " + std::to_string(r) + " outside a world of " + std::to_string(w));
    const double limit = timeout_s();

    // this rank's device (the local rank's when the launcher names one)
    Hello me{};
    me.magic = kMagic;
    me.rank = r;
    me.world = w;
    int ndev = 0;
    const bool gpu = cudaGetDeviceCount(&ndev) == cudaSuccess && ndev > 0;
    if (!gpu) cudaGetLastError();
    if (gpu) {
        const char* dv = env_first({"TINYMD_DEVICE", "LOCAL_RANK", "OMPI_COMM_WORLD_LOCAL_RANK", "MPI_LOCALRANKID"});
        if (dv) cudaSetDevice(std::atoi(dv) % ndev);
        int dev = 0;
        cudaDeviceProp prop;
        if (cudaGetDevice(&dev) == cudaSuccess && cudaGetDeviceProperties(&prop, dev) == cudaSuccess)
            std::memcpy(me.uuid, prop.uuid.bytes, 16);
        cudaGetLastError();
    }
    const char* mode = std::getenv("TINYMD_COMM");
    const std::string m = mode ? mode : "auto";
    if (m != "auto" && m != "socket" && m != "nccl") return fail("TINYMD_COMM must be auto, socket or nccl");
    me.nccl_ok = (gpu && m != "socket" && g_nccl.open()) ? 1 : 0;

    const char* host = env_first({"TINYMD_ADDR", "MASTER_ADDR"});
    uint32_t ip0 = 0;
    if (!resolve(host ? host : "127.0.0.1", &ip0)) return fail(std::string("cannot resolve ") + (host ? host : ""));
    int port = 29417;
    if (const char* p = std::getenv("TINYMD_PORT")) port = std::atoi(p);
    else if (const char* p = std::getenv("MASTER_PORT")) port = std::atoi(p) + 17;  // beside torch's store
    if (port <= 0 || port > 65535) return fail("bad TINYMD_PORT");

    fd_.assign(w, -1);
    uint16_t myport = 0;
    const int lfd = listen_on(r == 0 ? (uint16_t)port : 0, &myport);
    if (lfd < 0) return fail("cannot listen on a TCP port (rank " + std::to_string(r) + ")");
    me.port = myport;
    std::vector<Entry> table(w);
    uint8_t use_nccl = 0;
    ncclUniqueId uid{};
    bool ok = true;
    if (r == 0) {
        // rank 0: every other rank connects to the published port first
        std::vector<Hello> hs(w);
        hs[0] = me;
        for (int k = 1; k < w && ok; ++k) {
            uint32_t pip = 0;
            const int fd = accept_one(lfd, limit, &pip);
            Hello h{};
            if (fd < 0 || !io_all(fd, &h, sizeof(h), false, limit) || h.magic != kMagic || h.world != w ||
                h.rank <= 0 || h.rank >= w || fd_[h.rank] >= 0) {
                if (fd >= 0) close(fd);
                ok = false;
                break;
            }
            fd_[h.rank] = fd;
            hs[h.rank] = h;
            table[h.rank].ip = pip;
            table[h.rank].port = h.port;
        }
        if (!ok) {
            close(lfd);
            finalize();
            return fail("ranks did not all connect to rank 0 (port " + std::to_string(port) + ")");
        }
        // NCCL when every rank has it and its own device
        bool all = true, distinct = true;
        static const uint8_t zero[16] = {};
        for (int a = 0; a < w; ++a) {
            all = all && hs[a].nccl_ok && std::memcmp(hs[a].uuid, zero, 16) != 0;
            for (int b = 0; b < a; ++b) distinct = distinct && std::memcmp(hs[a].uuid, hs[b].uuid, 16) != 0;
        }
        use_nccl = (m != "socket" && all && distinct) ? 1 : 0;
        if (m == "nccl" && !use_nccl) use_nccl = 2;  // asked for and impossible: every rank fails
        if (use_nccl == 1 && g_nccl.get_unique_id(&uid) != ncclSuccess) use_nccl = 2;
        for (int k = 1; k < w && ok; ++k) {
            ok = io_all(fd_[k], &use_nccl, 1, true, limit) && io_all(fd_[k], table.data(), sizeof(Entry) * w, true, limit);
            if (ok && use_nccl == 1) ok = io_all(fd_[k], &uid, sizeof(uid), true, limit);
        }
    } else {
        const int fd = connect_to(ip0, (uint16_t)port, limit);
        ok = fd >= 0 && io_all(fd, &me, sizeof(me), true, limit) && io_all(fd, &use_nccl, 1, false, limit) &&
             io_all(fd, table.data(), sizeof(Entry) * w, false, limit);
        if (ok && use_nccl == 1) ok = io_all(fd, &uid, sizeof(uid), false, limit);
        if (fd >= 0) fd_[0] = fd;
        // the mesh: connect to every rank between 0 and this one, accept the higher ones
        for (int k = 1; k < r && ok; ++k) {
            const int c = connect_to(table[k].ip, table[k].port, limit);
            int32_t who = r;
            ok = c >= 0 && io_all(c, &who, sizeof(who), true, limit);
            if (c >= 0) fd_[k] = c;
        }
        for (int k = r + 1; k < w && ok; ++k) {
            const int c = accept_one(lfd, limit, nullptr);
            int32_t who = -1;
            ok = c >= 0 && io_all(c, &who, sizeof(who), false, limit) && who > r && who < w && fd_[who] < 0;
            if (ok) fd_[who] = c;
            else if (c >= 0) close(c);
        }
    }
    close(lfd);
    if (!ok) {
        finalize();
        return fail("the TCP mesh between the ranks could not be completed (rank " + std::to_string(r) + ")");
    }
    if (use_nccl == 2) {
        finalize();
        return fail("TINYMD_COMM=nccl needs libnccl.so.2 and a distinct GPU on every rank");
    }
    world_ = w;
    rank_ = r;
    topo_set = false;  // a layout made before the ranks connected was a one-rank layout
    if (use_nccl == 1) {
        ncclComm_t c = nullptr;
        const ncclResult_t e = g_nccl.init_rank(&c, w, uid, r);
        if (e != ncclSuccess) {
            finalize();
            return fail(std::string("ncclCommInitRank: ") + g_nccl.error_string(e));
        }
        nccl_ = c;
    }
    return barrier();
}

void Comm::finalize() {
    if (nccl_) {
        g_nccl.destroy(static_cast<ncclComm_t>(nccl_));
        nccl_ = nullptr;
    }
    for (int& fd : fd_)
        if (fd >= 0) {
            close(fd);
            fd = -1;
        }
    fd_.clear();
    world_ = 1;
    rank_ = 0;
    topo_set = false;
}

bool Comm::exchange(const std::vector<HostMsg>& sends, const std::vector<HostMsg>& recvs) {
    struct X {
        int fd;
        char* p;
        size_t left;
    };
    std::vector<X> tx, rx;
    // one message per peer and direction: two on one connection would interleave their bytes
    std::vector<char> seen_tx(world_, 0), seen_rx(world_, 0);
    for (const HostMsg& s : sends) {
        if (s.peer < 0 || s.peer >= world_ || s.peer == rank_ || seen_tx[s.peer]++) return fail("exchange: bad peer");
        if (s.bytes) tx.push_back({fd_[s.peer], static_cast<char*>(s.data), s.bytes});
    }
    for (const HostMsg& s : recvs) {
        if (s.peer < 0 || s.peer >= world_ || s.peer == rank_ || seen_rx[s.peer]++) return fail("exchange: bad peer");
        if (s.bytes) rx.push_back({fd_[s.peer], static_cast<char*>(s.data), s.bytes});
    }
    const double limit = timeout_s();
    double last = now_s();
    std::vector<pollfd> pf;
    while (!tx.empty() || !rx.empty()) {
        pf.clear();
        for (const X& x : tx) pf.push_back({x.fd, POLLOUT, 0});
        for (const X& x : rx) pf.push_back({x.fd, POLLIN, 0});
        const int n = poll(pf.data(), (nfds_t)pf.size(), 500);
        if (n < 0) {
            if (errno == EINTR) continue;
            return fail("exchange: poll failed");
        }
        if (n == 0) {
            if (now_s() - last > limit) return fail("exchange: no progress from a peer rank (timed out)");
            continue;
        }
        for (size_t i = 0; i < tx.size(); ++i) {
            const short ev = pf[i].revents;
            if (ev & POLLOUT) {
                const ssize_t k = ::send(tx[i].fd, tx[i].p, tx[i].left, MSG_NOSIGNAL | MSG_DONTWAIT);
                if (k > 0) {
                    tx[i].p += k;
                    tx[i].left -= (size_t)k;
                    last = now_s();
                } else if (k < 0 && errno != EAGAIN && errno != EWOULDBLOCK && errno != EINTR) {
                    return fail("exchange: a peer rank closed its connection");
                }
            } else if (ev & (POLLERR | POLLHUP | POLLNVAL)) {
                return fail("exchange: a peer rank closed its connection");
            }
        }
        for (size_t i = 0; i < rx.size(); ++i) {
            const short ev = pf[tx.size() + i].revents;
            if (ev & POLLIN) {
                const ssize_t k = ::recv(rx[i].fd, rx[i].p, rx[i].left, MSG_DONTWAIT);
                if (k > 0) {
                    rx[i].p += k;
                    rx[i].left -= (size_t)k;
                    last = now_s();
                } else if (k == 0 || (errno != EAGAIN && errno != EWOULDBLOCK && errno != EINTR)) {
                    return fail("exchange: a peer rank closed its connection");
                }
            } else if (ev & (POLLERR | POLLHUP | POLLNVAL)) {
                return fail("exchange: a peer rank closed its connection");
            }
        }
        tx.erase(std::remove_if(tx.begin(), tx.end(), [](const X& x) { return x.left == 0; }), tx.end());
        rx.erase(std::remove_if(rx.begin(), rx.end(), [](const X& x) { return x.left == 0; }), rx.end());
    }
    return true;
}

bool Comm::exchange_device(const std::vector<HostMsg>& sends, const std::vector<HostMsg>& recvs,
                           cudaStream_t stream) {
    if (!nccl_) return fail("exchange_device: no NCCL communicator");
    ncclComm_t c = static_cast<ncclComm_t>(nccl_);
    ncclResult_t e = g_nccl.group_start();
    for (const HostMsg& s : sends)
        if (e == ncclSuccess && s.bytes) e = g_nccl.send(s.data, s.bytes, ncclChar, s.peer, c, stream);
    for (const HostMsg& s : recvs)
        if (e == ncclSuccess && s.bytes) e = g_nccl.recv(s.data, s.bytes, ncclChar, s.peer, c, stream);
    const ncclResult_t e2 = g_nccl.group_end();
    if (e == ncclSuccess) e = e2;
    if (e != ncclSuccess) return fail(std::string("NCCL send/recv: ") + g_nccl.error_string(e));
    return true;
}

template <class T, class Op>
bool Comm::allreduce(T* v, int n, Op op) {
    if (world_ <= 1 || n <= 0) return true;
    const size_t bytes = sizeof(T) * (size_t)n;
    if (rank_ == 0) {
        std::vector<T> all((size_t)world_ * n);
        std::vector<HostMsg> rx;
        for (int r = 1; r < world_; ++r) rx.push_back({r, &all[(size_t)r * n], bytes});
        if (!exchange({}, rx)) return false;
        for (int i = 0; i < n; ++i) {
            T acc = v[i];
            for (int r = 1; r < world_; ++r) acc = op(acc, all[(size_t)r * n + i]);
            v[i] = acc;
        }
        std::vector<HostMsg> tx;
        for (int r = 1; r < world_; ++r) tx.push_back({r, v, bytes});
        return exchange(tx, {});
    }
    return exchange({{0, v, bytes}}, {}) && exchange({}, {{0, v, bytes}});
}

bool Comm::allreduce_sum(double* v, int n) { return allreduce(v, n, [](double a, double b) { return a + b; }); }
bool Comm::allreduce_max(double* v, int n) { return allreduce(v, n, [](double a, double b) { return a > b ? a : b; }); }
bool Comm::allreduce_sum(long long* v, int n) {
    return allreduce(v, n, [](long long a, long long b) { return a + b; });
}
bool Comm::barrier() {
    long long one = 1;
    return allreduce_sum(&one, 1) && (world_ <= 1 || one == world_ || fail("barrier: rank count mismatch"));
}

}  // namespace tmd

// ---- C entry points of the rank layout and transport (tests and non-C++ callers) ----------------
extern "C" {

int tmd_node_config(int world, double const* len, int* dims) {
    if (world < 1) return -1;
    tmd::node_config(world, len, dims);
    return 0;
}

// peer[26], shift[26*3], *selfmask of `rank` in a world of dims[0]*dims[1]*dims[2] ranks
int tmd_topology(int rank, int const* dims, int* peer, int* shift, unsigned* selfmask) {
    const int world = dims[0] * dims[1] * dims[2];
    if (world < 1 || rank < 0 || rank >= world) return -1;
    tmd::Topology t;
    tmd::make_topology(world, rank, dims, t);
    for (int k = 0; k < 26; ++k) {
        peer[k] = t.peer[k];
        for (int d = 0; d < 3; ++d) shift[3 * k + d] = t.shift[k][d];
    }
    *selfmask = t.selfmask;
    return 0;
}

const char* tmd_comm_transport(void) { return tmd::comm().transport(); }

// The NCCL binding on this process's GPU alone: a one-rank communicator sends `bytes` of a device
// buffer to itself through the same group / send / receive calls the halo exchange issues, on a
// stream, and the copy is compared.  0 when it matches, -2 without libnccl, -1 otherwise.
int tmd_comm_nccl_selftest(long long bytes) {
    using tmd::g_nccl;
    if (bytes <= 0 || !g_nccl.open()) return bytes <= 0 ? -1 : -2;
    ncclUniqueId id;
    ncclComm_t c = nullptr;
    if (g_nccl.get_unique_id(&id) != ncclSuccess || g_nccl.init_rank(&c, 1, id, 0) != ncclSuccess) return -1;
    const size_t n = (size_t)bytes;
    std::vector<unsigned char> h(n), back(n, 0);
    for (size_t i = 0; i < n; ++i) h[i] = (unsigned char)(i * 131u + 7u);
    void *a = nullptr, *b = nullptr;
    cudaStream_t st = nullptr;
    bool ok = cudaMalloc(&a, n) == cudaSuccess && cudaMalloc(&b, n) == cudaSuccess &&
              cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) == cudaSuccess &&
              cudaMemcpy(a, h.data(), n, cudaMemcpyHostToDevice) == cudaSuccess &&
              cudaMemset(b, 0, n) == cudaSuccess;
    if (ok) {
        ncclResult_t e = g_nccl.group_start();
        if (e == ncclSuccess) e = g_nccl.send(a, n, ncclChar, 0, c, st);
        if (e == ncclSuccess) e = g_nccl.recv(b, n, ncclChar, 0, c, st);
        const ncclResult_t e2 = g_nccl.group_end();
        ok = e == ncclSuccess && e2 == ncclSuccess && cudaStreamSynchronize(st) == cudaSuccess &&
             cudaMemcpy(back.data(), b, n, cudaMemcpyDeviceToHost) == cudaSuccess && back == h;
    }
    g_nccl.destroy(c);
    if (st) cudaStreamDestroy(st);
    if (a) cudaFree(a);
    if (b) cudaFree(b);
    cudaGetLastError();
    return ok ? 0 : -1;
}

int tmd_comm_allreduce_sum(double* v, int n) { return tmd::comm().allreduce_sum(v, n) ? 0 : -1; }

// one message to `to` and one from `from` (host buffers)
int tmd_comm_sendrecv(int to, void const* sbuf, long long sbytes, int from, void* rbuf, long long rbytes) {
    std::vector<tmd::HostMsg> tx, rx;
    if (sbytes > 0) tx.push_back({to, const_cast<void*>(sbuf), (size_t)sbytes});
    if (rbytes > 0) rx.push_back({from, rbuf, (size_t)rbytes});
    return tmd::comm().exchange(tx, rx) ? 0 : -1;
}

}  // extern "C"
