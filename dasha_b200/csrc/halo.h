// halo.h -- z-slab decomposition of one periodic-x/y grid over several contexts (one per GPU),
// the multi-GPU form of the reference's 2-D (x, z) MPI decomposition (mhd01.for:5-6) with its
// 2-plane halo exchange message4 (t3dsdsc.f:6354-6419), restricted to z.
//
// The interior rows 2..mz-3 of the global grid are split into n slabs of consecutive rows.
// Slab s owns rows first .. first+count-1; its context is an ordinary context over the local
// grid of rows first-2 .. first+count+1 (mzl = count + 4 planes), so every kernel computes
// exactly its own rows.  At an end that is a global wall the two outer planes are the
// reference's wall rows and the kernels write them as in the one-domain run.  At an end shared
// with a neighbour the kernels write the wall rule into the two ghost planes as well, but the
// engine refreshes them from the neighbour (its two own planes next to the cut) after every
// launch whose output a later launch reads at z-neighbours and before that read: the ghost
// planes of a field are never read between a write and the exchange that follows it.
//
// Two exchanges implement it:
//   HaloLocal  every slab in this process (one host thread per slab while a group call runs):
//              each slab copies its neighbours' edge planes into its ghost planes
//              (cudaMemcpyPeerAsync, NVLink between GPUs), ordered against the neighbours'
//              launches by events its stream waits on (no host synchronisation).
//   HaloNccl   one process per GPU: ncclSend / ncclRecv of the edge planes of each field in one
//              NCCL group on the context's stream (no host synchronisation), and the dt
//              reduction of setdt as ncclAllReduce.  NCCL is opened at run time (dlopen), so
//              the library has no link-time dependency on it.
// Both move the same planes: SlabGeom's send_* / recv_* give their byte offsets in a field.
#pragma once

#include <cuda_runtime.h>
#include <nccl.h>   // types only: the library itself is opened at run time
#include <dlfcn.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstring>
#include <limits>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

namespace dasha {

// rows first .. first+count-1 of the global grid are slab s's own
struct SlabPart {
    int first = 0, count = 0;
};

// The partition of the interior rows 2..mz-3 into n slabs: count = rows / n, the first rows % n
// slabs one more (every slab at least 3 rows, so that a local grid is at least the smallest
// accepted one, mz = 7, and the two edge planes a neighbour reads are own rows).
inline bool slab_partition(int mz, int n, int s, SlabPart& out) {
    const int rows = mz - 4;
    if (n < 1 || s < 0 || s >= n || rows < 3 * n) return false;
    const int base = rows / n, extra = rows % n;
    out.first = 2 + s * base + std::min(s, extra);
    out.count = base + (s < extra ? 1 : 0);
    return true;
}

// The geometry of one slab's exchange: the local grid has mzl planes of sz nodes.
struct SlabGeom {
    int n = 1, s = 0, mzl = 0, device = 0;
    int zfirst = 2, mzg = 0;      // the first own row and the plane count of the global grid
    long sz = 0;
    size_t elem = 0;
    cudaStream_t st = nullptr;
    const void* pool = nullptr;   // the field pool: field q at pool + q * fbytes
    size_t fbytes = 0;
    bool lower() const { return s > 0; }
    bool upper() const { return s < n - 1; }
    size_t plane_bytes() const { return (size_t)sz * elem; }
    // byte offsets in a field: the two planes sent down / up and the two ghost planes filled
    // from below / above
    size_t send_lo() const { return 2 * plane_bytes(); }
    size_t send_hi() const { return (size_t)(mzl - 4) * plane_bytes(); }
    size_t recv_lo() const { return 0; }
    size_t recv_hi() const { return (size_t)(mzl - 2) * plane_bytes(); }
    size_t span() const { return 2 * plane_bytes(); }
};

struct Halo {
    SlabGeom geo;
    std::string err;
    virtual ~Halo() = default;
    // refreshes the ghost planes of the nf fields f (field pointers of this slab's pool) on the
    // slab's stream; false (and err) when the exchange failed
    virtual bool exchange(void* const* f, int nf) = 0;
    // the group's minimum dt and maximum flag, from this slab's values (a NaN dt wins)
    virtual bool reduce(double* dt, int* flag) = 0;
    // the group's diagnostics from this slab's (sums of [0..2], maxima of [3], [5], [7], minima
    // of [4], [6], [8]) and the maximum blow-up flag
    virtual bool reduce_diag(double* out9, int* flag) = 0;
    // true when each slab runs in its own process (the entry points of one context are called
    // per process); false for a group of slabs driven by the group entry points
    virtual bool per_process() const = 0;
};

// ---- the slabs of one process ----

// A barrier of n host threads with a time limit: a member that fails or never arrives makes
// every waiter return false instead of waiting for ever.
class GroupBarrier {
public:
    explicit GroupBarrier(int n) : n_(n) {}
    bool arrive(double limit_s) {
        std::unique_lock<std::mutex> lk(m_);
        if (failed_) return false;
        const long g = gen_;
        if (++count_ == n_) {
            count_ = 0;
            ++gen_;
            cv_.notify_all();
            return true;
        }
        const bool done = cv_.wait_for(lk, std::chrono::duration<double>(limit_s), [&] { return gen_ != g || failed_; });
        if (!done) {
            failed_ = true;
            cv_.notify_all();
            return false;
        }
        return gen_ != g;
    }
    void fail() {
        std::lock_guard<std::mutex> lk(m_);
        failed_ = true;
        cv_.notify_all();
    }
    bool failed() {
        std::lock_guard<std::mutex> lk(m_);
        return failed_;
    }
    void reset() {
        std::lock_guard<std::mutex> lk(m_);
        failed_ = false;
        count_ = 0;
    }

private:
    std::mutex m_;
    std::condition_variable cv_;
    int n_, count_ = 0;
    long gen_ = 0;
    bool failed_ = false;
};

struct LocalGroup {
    explicit LocalGroup(int n) : bar(n), members(n, nullptr), wr(n, nullptr), cp(n, nullptr) {}
    ~LocalGroup() {
        for (cudaEvent_t e : wr) if (e) cudaEventDestroy(e);
        for (cudaEvent_t e : cp) if (e) cudaEventDestroy(e);
    }
    GroupBarrier bar;
    std::vector<const SlabGeom*> members;   // slab s's geometry
    // slab s's events: its writes before an exchange, its ghost copies of an exchange (each
    // slab records only its own; the others read them after a barrier)
    std::vector<cudaEvent_t> wr, cp;
    double limit_s = 300.0;                 // a barrier wait longer than this fails the group call
};

class HaloLocal : public Halo {
public:
    explicit HaloLocal(std::shared_ptr<LocalGroup> g) : grp(std::move(g)) {}
    std::shared_ptr<LocalGroup> grp;

    bool per_process() const override { return false; }

    // Stream order, no host synchronisation: the copies wait (cudaStreamWaitEvent) on the
    // neighbours' writes, and this slab's next launches on the neighbours' copies out of its edge
    // planes; the host barriers only order each event's record before the waits on it.
    bool exchange(void* const* f, int nf) override {
        if (grp->bar.failed()) return fail("an earlier exchange of the group failed");
        const int s = geo.s;
        if (!grp->wr[s] && (cudaEventCreateWithFlags(&grp->wr[s], cudaEventDisableTiming) != cudaSuccess ||
                            cudaEventCreateWithFlags(&grp->cp[s], cudaEventDisableTiming) != cudaSuccess))
            return fail("event creation failed");
        if (cudaEventRecord(grp->wr[s], geo.st) != cudaSuccess) return fail("event record failed");
        if (!grp->bar.arrive(grp->limit_s)) return fail("a slab of the group did not reach the exchange");
        if ((geo.lower() && !grp->members[s - 1]) || (geo.upper() && !grp->members[s + 1]))
            return fail("a neighbouring slab of the group was destroyed");
        if (geo.lower() && cudaStreamWaitEvent(geo.st, grp->wr[s - 1], 0) != cudaSuccess) return fail("event wait failed");
        if (geo.upper() && cudaStreamWaitEvent(geo.st, grp->wr[s + 1], 0) != cudaSuccess) return fail("event wait failed");
        for (int q = 0; q < nf; ++q) {
            const size_t off = (size_t)((const char*)f[q] - (const char*)geo.pool);
            if ((const char*)f[q] < (const char*)geo.pool || off % geo.fbytes != 0) return fail("field outside the pool");
            const size_t idx = off / geo.fbytes;
            char* dst = (char*)f[q];
            if (geo.lower()) {
                const SlabGeom& o = *grp->members[s - 1];
                const char* src = (const char*)o.pool + idx * o.fbytes + o.send_hi();
                if (cudaMemcpyPeerAsync(dst + geo.recv_lo(), geo.device, src, o.device, geo.span(), geo.st) != cudaSuccess)
                    return fail("ghost copy from the lower slab failed");
            }
            if (geo.upper()) {
                const SlabGeom& o = *grp->members[s + 1];
                const char* src = (const char*)o.pool + idx * o.fbytes + o.send_lo();
                if (cudaMemcpyPeerAsync(dst + geo.recv_hi(), geo.device, src, o.device, geo.span(), geo.st) != cudaSuccess)
                    return fail("ghost copy from the upper slab failed");
            }
        }
        if (cudaEventRecord(grp->cp[s], geo.st) != cudaSuccess) return fail("event record failed");
        if (!grp->bar.arrive(grp->limit_s)) return fail("a slab of the group did not finish the exchange");
        // the neighbours' copies out of this slab's edge planes end before its next launch
        if (geo.lower() && cudaStreamWaitEvent(geo.st, grp->cp[s - 1], 0) != cudaSuccess) return fail("event wait failed");
        if (geo.upper() && cudaStreamWaitEvent(geo.st, grp->cp[s + 1], 0) != cudaSuccess) return fail("event wait failed");
        return true;
    }
    bool reduce(double*, int*) override { return true; }   // the group entry points reduce on the host
    bool reduce_diag(double*, int*) override { return true; }

private:
    bool fail(const char* m) {
        err = m;
        grp->bar.fail();
        return false;
    }
};

// ---- one slab per process: NCCL ----

struct NcclApi {
    decltype(&ncclGetUniqueId) get_unique_id = nullptr;
    decltype(&ncclCommInitRank) comm_init_rank = nullptr;
    decltype(&ncclCommDestroy) comm_destroy = nullptr;
    decltype(&ncclGroupStart) group_start = nullptr;
    decltype(&ncclGroupEnd) group_end = nullptr;
    decltype(&ncclSend) send = nullptr;
    decltype(&ncclRecv) recv = nullptr;
    decltype(&ncclAllReduce) all_reduce = nullptr;
    decltype(&ncclGetErrorString) error_string = nullptr;
    std::string why;
    bool ok() const { return send != nullptr; }
    // The process's NCCL: the libnccl.so.2 already loaded (torch's, for instance), else the one
    // the loader finds.  A process holds one object of that name, and a library loaded later
    // that needs libnccl.so.2 binds to it: a process that also uses torch imports torch first.
    static const NcclApi& get() {
        static NcclApi api = [] {
            NcclApi a;
            void* h = dlopen("libnccl.so.2", RTLD_NOW | RTLD_NOLOAD);
            if (!h) h = dlopen("libnccl.so.2", RTLD_NOW | RTLD_LOCAL);
            if (!h) h = dlopen("libnccl.so", RTLD_NOW | RTLD_LOCAL);
            if (!h) { a.why = std::string("libnccl.so.2 not found: ") + (dlerror() ? dlerror() : ""); return a; }
            auto sym = [&](const char* n) { return dlsym(h, n); };
            a.get_unique_id = (decltype(a.get_unique_id))sym("ncclGetUniqueId");
            a.comm_init_rank = (decltype(a.comm_init_rank))sym("ncclCommInitRank");
            a.comm_destroy = (decltype(a.comm_destroy))sym("ncclCommDestroy");
            a.group_start = (decltype(a.group_start))sym("ncclGroupStart");
            a.group_end = (decltype(a.group_end))sym("ncclGroupEnd");
            a.all_reduce = (decltype(a.all_reduce))sym("ncclAllReduce");
            a.error_string = (decltype(a.error_string))sym("ncclGetErrorString");
            a.recv = (decltype(a.recv))sym("ncclRecv");
            a.send = (decltype(a.send))sym("ncclSend");
            if (!a.get_unique_id || !a.comm_init_rank || !a.comm_destroy || !a.group_start || !a.group_end ||
                !a.all_reduce || !a.recv || !a.send) {
                a.send = nullptr;
                a.why = "libnccl.so.2 lacks a symbol of the halo exchange";
            }
            return a;
        }();
        return api;
    }
};

class HaloNccl : public Halo {
public:
    ~HaloNccl() override {
        if (comm) NcclApi::get().comm_destroy(comm);
        if (dbuf) cudaFree(dbuf);
        if (hbuf) cudaFreeHost(hbuf);
    }
    // joins the communicator of the n slabs (collective: every rank calls it with the same id)
    bool init(const ncclUniqueId& id) {
        const NcclApi& a = NcclApi::get();
        if (!a.ok()) { err = a.why; return false; }
        if (cudaMalloc(&dbuf, 10 * sizeof(double)) != cudaSuccess || cudaMallocHost(&hbuf, 10 * sizeof(double)) != cudaSuccess) {
            err = "device or pinned buffer of the dt reduction";
            return false;
        }
        ncclResult_t r = a.comm_init_rank(&comm, geo.n, id, geo.s);
        if (r != ncclSuccess) { comm = nullptr; return nccl_fail("ncclCommInitRank", r); }
        return true;
    }
    bool per_process() const override { return true; }

    bool exchange(void* const* f, int nf) override {
        const NcclApi& a = NcclApi::get();
        if (!comm) { err = "no NCCL communicator"; return false; }
        if (!geo.lower() && !geo.upper()) return true;   // one slab: its outer planes are walls
        ncclResult_t r = a.group_start();
        if (r != ncclSuccess) return nccl_fail("ncclGroupStart", r);
        for (int q = 0; q < nf && r == ncclSuccess; ++q) {
            char* b = (char*)f[q];
            if (geo.lower()) {
                r = a.send(b + geo.send_lo(), geo.span(), ncclInt8, geo.s - 1, comm, geo.st);
                if (r == ncclSuccess) r = a.recv(b + geo.recv_lo(), geo.span(), ncclInt8, geo.s - 1, comm, geo.st);
            }
            if (geo.upper() && r == ncclSuccess) {
                r = a.send(b + geo.send_hi(), geo.span(), ncclInt8, geo.s + 1, comm, geo.st);
                if (r == ncclSuccess) r = a.recv(b + geo.recv_hi(), geo.span(), ncclInt8, geo.s + 1, comm, geo.st);
            }
        }
        ncclResult_t e = a.group_end();
        if (r != ncclSuccess) return nccl_fail("ncclSend/ncclRecv", r);
        if (e != ncclSuccess) return nccl_fail("ncclGroupEnd", e);
        return true;
    }

    bool reduce(double* dt, int* flag) override {
        const NcclApi& a = NcclApi::get();
        if (!comm) { err = "no NCCL communicator"; return false; }
        // a NaN dt travels as -inf (the minimum) and comes back as NaN
        hbuf[0] = std::isnan(*dt) ? -std::numeric_limits<double>::infinity() : *dt;
        int fl = *flag;
        std::memcpy(hbuf + 1, &fl, sizeof(int));
        if (cudaMemcpyAsync(dbuf, hbuf, 16, cudaMemcpyHostToDevice, geo.st) != cudaSuccess) { err = "dt upload"; return false; }
        ncclResult_t r = a.group_start();
        if (r == ncclSuccess) r = a.all_reduce(dbuf, dbuf, 1, ncclFloat64, ncclMin, comm, geo.st);
        if (r == ncclSuccess) r = a.all_reduce(dbuf + 1, dbuf + 1, 1, ncclInt32, ncclMax, comm, geo.st);
        ncclResult_t e = a.group_end();
        if (r != ncclSuccess) return nccl_fail("ncclAllReduce", r);
        if (e != ncclSuccess) return nccl_fail("ncclGroupEnd", e);
        if (cudaMemcpyAsync(hbuf, dbuf, 16, cudaMemcpyDeviceToHost, geo.st) != cudaSuccess ||
            cudaStreamSynchronize(geo.st) != cudaSuccess) {
            err = "dt download";
            return false;
        }
        *dt = std::isinf(hbuf[0]) && hbuf[0] < 0 ? std::numeric_limits<double>::quiet_NaN() : hbuf[0];
        std::memcpy(&fl, hbuf + 1, sizeof(int));
        *flag = fl;
        return true;
    }

    bool reduce_diag(double* out9, int* flag) override {
        const NcclApi& a = NcclApi::get();
        if (!comm) { err = "no NCCL communicator"; return false; }
        // [0..2] summed, the maxima as they are, the minima negated (one max), the flag as a double
        for (int q = 0; q < 3; ++q) hbuf[q] = out9[q];
        for (int q = 0; q < 3; ++q) { hbuf[3 + q] = out9[3 + 2 * q]; hbuf[6 + q] = -out9[4 + 2 * q]; }
        hbuf[9] = (double)*flag;
        if (cudaMemcpyAsync(dbuf, hbuf, 10 * sizeof(double), cudaMemcpyHostToDevice, geo.st) != cudaSuccess) {
            err = "diagnostics upload";
            return false;
        }
        ncclResult_t r = a.group_start();
        if (r == ncclSuccess) r = a.all_reduce(dbuf, dbuf, 3, ncclFloat64, ncclSum, comm, geo.st);
        if (r == ncclSuccess) r = a.all_reduce(dbuf + 3, dbuf + 3, 7, ncclFloat64, ncclMax, comm, geo.st);
        ncclResult_t e = a.group_end();
        if (r != ncclSuccess) return nccl_fail("ncclAllReduce", r);
        if (e != ncclSuccess) return nccl_fail("ncclGroupEnd", e);
        if (cudaMemcpyAsync(hbuf, dbuf, 10 * sizeof(double), cudaMemcpyDeviceToHost, geo.st) != cudaSuccess ||
            cudaStreamSynchronize(geo.st) != cudaSuccess) {
            err = "diagnostics download";
            return false;
        }
        for (int q = 0; q < 3; ++q) out9[q] = hbuf[q];
        for (int q = 0; q < 3; ++q) { out9[3 + 2 * q] = hbuf[3 + q]; out9[4 + 2 * q] = -hbuf[6 + q]; }
        *flag = hbuf[9] != 0.0;
        return true;
    }

private:
    ncclComm_t comm = nullptr;
    double* dbuf = nullptr;
    double* hbuf = nullptr;
    bool nccl_fail(const char* what, ncclResult_t r) {
        const NcclApi& a = NcclApi::get();
        err = std::string(what) + " failed: " + (a.error_string ? a.error_string(r) : std::to_string((int)r));
        return false;
    }
};

}  // namespace dasha
