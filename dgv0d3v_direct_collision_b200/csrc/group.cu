// group.cu -- one batch of VDFs on several velocity grids as one graph launch.
//
// A mixed batch (VDFs of different grids, one context per grid, all on one
// device) is evaluated by forking from an origin stream to each member
// context's stream, running that context's collision path there
// (EvalCollisionPeriodicAPlus_DGV, collision_mod.f90:143-229, for every VDF of
// the member) and joining back.  The first call for a given member list runs
// eagerly (it settles autotuned chunk counts, work lists and buffers); the
// second captures the whole fork/join into one CUDA graph; later calls replay
// it with a single launch.  The members' kernels may overlap on the device.
// On the tensor cores (block form, same nodes per cell and VDF tile size, at
// most four members) the captured graph holds three kernels for all members
// -- the f preparation, one persistent collision kernel, the final step --
// instead of several launches per member and block set.
#include <cstring>
#include <map>
#include <mutex>
#include <vector>

#include "dgv_internal.h"

namespace dgv {

int collide_device(Ctx *c, const double *d_f, double *d_q, int nvdf, int precision, double scale);
int collide_tc2_group(Ctx *const *cs, const double *const *f, double *const *q, const int *nb, int n,
                      cudaStream_t origin, cudaEvent_t fork2, const cudaEvent_t *join);

namespace {

struct Member {
    Ctx *c;
    const double *f;
    double *q;
    int nb;
    int project;
    bool operator<(const Member &o) const { return std::memcmp(this, &o, sizeof(*this)) < 0; }
};

struct GroupKey {
    std::vector<Member> m;
    cudaStream_t origin;
    int precision;
    bool operator<(const GroupKey &o) const
    {
        if (precision != o.precision) return precision < o.precision;
        if (origin != o.origin) return origin < o.origin;
        return m < o.m;
    }
};

struct GroupGraph {
    int calls = 0;
    cudaGraphExec_t exec = nullptr;
    std::vector<long long> launches;  // per member, counted while capturing
};

std::map<GroupKey, GroupGraph> g_groups;
std::recursive_mutex g_groups_mu;

// fork from origin to every member stream, run the members, join back; with
// `persistent`, members on the tensor cores' block form that can share one
// launch are served by one persistent kernel (collide_tc2_group)
int run_members(const GroupKey &k, cudaEvent_t fork, cudaEvent_t fork2, std::vector<cudaEvent_t> &join,
                bool persistent)
{
    Ctx *c0 = k.m[0].c;
    if (persistent && k.precision == DGV_PREC_TC && k.m.size() <= 4) {
        std::vector<Ctx *> cs;
        std::vector<const double *> fs;
        std::vector<double *> qs;
        std::vector<int> nbs;
        bool proj_ok = true;
        for (const Member &mb : k.m) {
            cs.push_back(mb.c);
            fs.push_back(mb.f);
            qs.push_back(mb.q);
            nbs.push_back(mb.nb);
            proj_ok = proj_ok && (mb.project != 0) == mb.c->project;
        }
        if (proj_ok) {
            const int rc = collide_tc2_group(cs.data(), fs.data(), qs.data(), nbs.data(), (int)cs.size(), k.origin,
                                             fork2, join.data());
            if (rc != DGV_EUNSUP) return rc;
            c0->err.clear();  // members that cannot share a launch: one call per member
        }
    }
    DGV_CUDA(c0, cudaEventRecord(fork, k.origin));
    for (size_t i = 0; i < k.m.size(); i++) {
        const Member &mb = k.m[i];
        Ctx *c = mb.c;
        if (c->stream != k.origin) DGV_CUDA(c, cudaStreamWaitEvent(c->stream, fork, 0));
        int rc = collide_device(c, mb.f, mb.q, mb.nb, k.precision, 1.0);
        if (rc) return rc;
        if (c->stream != k.origin) {
            DGV_CUDA(c, cudaEventRecord(join[i], c->stream));
            DGV_CUDA(c, cudaStreamWaitEvent(k.origin, join[i], 0));
        }
    }
    return DGV_OK;
}

struct Events {
    cudaEvent_t fork = nullptr, fork2 = nullptr;
    std::vector<cudaEvent_t> join;
    ~Events()
    {
        if (fork) cudaEventDestroy(fork);
        if (fork2) cudaEventDestroy(fork2);
        for (cudaEvent_t e : join)
            if (e) cudaEventDestroy(e);
    }
};

}  // namespace

// drops every group graph that has c as a member (its buffers or A-arrays changed)
void release_group_graphs(const Ctx *c)
{
    std::lock_guard<std::recursive_mutex> lk(g_groups_mu);
    for (auto it = g_groups.begin(); it != g_groups.end();) {
        bool hit = false;
        for (const Member &mb : it->first.m) hit = hit || mb.c == c;
        if (hit) {
            if (it->second.exec) cudaGraphExecDestroy(it->second.exec);
            it = g_groups.erase(it);
        } else {
            ++it;
        }
    }
}

}  // namespace dgv

using namespace dgv;

extern "C" int dgv_collide_group(int32_t n, dgv_ctx *const *ctxs, const int32_t *nb, const double *const *f,
                                 double *const *q, int precision, void *stream)
{
    if (n < 1 || !ctxs || !nb || !f || !q || !ctxs[0]) return DGV_EINVAL;
    Ctx *c0 = &ctxs[0]->c;
    c0->err.clear();
    GroupKey key;
    key.precision = precision;
    key.origin = stream ? (cudaStream_t)stream : c0->stream;
    for (int32_t i = 0; i < n; i++) {
        if (!ctxs[i]) return set_err(c0, DGV_EINVAL, "collide_group: NULL context");
        Ctx *c = &ctxs[i]->c;
        c->err.clear();
        if (c->device != c0->device) return set_err(c0, DGV_EINVAL, "collide_group: contexts on different devices");
        if (nb[i] < 1 || !f[i] || !q[i]) return set_err(c0, DGV_EINVAL, "collide_group: need nb >= 1 and arrays");
        bool fdev = false, qdev = false;
        if (classify_ptr(c, f[i], &fdev) || classify_ptr(c, q[i], &qdev) || !fdev || !qdev)
            return set_err(c0, DGV_EINVAL, "collide_group: f and q must be device pointers of the members' device");
        if (!c->lay.blk) return set_err(c0, DGV_ESTATE, "collide_group: a member has no A-arrays loaded");
        Member mb;
        std::memset(&mb, 0, sizeof(mb));
        mb.c = c; mb.f = f[i]; mb.q = q[i]; mb.nb = nb[i]; mb.project = c->project;
        key.m.push_back(mb);
    }
    DGV_CUDA(c0, cudaSetDevice(c0->device));
    Events ev;
    DGV_CUDA(c0, cudaEventCreateWithFlags(&ev.fork, cudaEventDisableTiming));
    DGV_CUDA(c0, cudaEventCreateWithFlags(&ev.fork2, cudaEventDisableTiming));
    ev.join.assign(2 * key.m.size(), nullptr);
    for (auto &e : ev.join) DGV_CUDA(c0, cudaEventCreateWithFlags(&e, cudaEventDisableTiming));

    // propagate a member's error message to the first context
    auto fail = [&](int rc) {
        for (const Member &mb : key.m)
            if (!mb.c->err.empty() && mb.c != c0) c0->err = mb.c->err;
        return rc;
    };
    {
        // entries are looked up again after running members: a buffer that
        // grows inside a member releases the group graphs holding its context
        std::unique_lock<std::recursive_mutex> lk(g_groups_mu);
        GroupGraph &gr = g_groups[key];
        if (gr.exec) {
            DGV_CUDA(c0, cudaGraphLaunch(gr.exec, key.origin));
            for (size_t i = 0; i < key.m.size(); i++) count_launches(key.m[i].c, gr.launches[i]);
        } else if (gr.calls++ == 0) {
            int rc = run_members(key, ev.fork, ev.fork2, ev.join, false);
            if (rc) return fail(rc);
        } else {
            std::vector<long long> before;
            for (const Member &mb : key.m) before.push_back(mb.c->kt_all);
            cudaGraph_t graph = nullptr;
            DGV_CUDA(c0, cudaStreamBeginCapture(key.origin, cudaStreamCaptureModeThreadLocal));
            int rc = run_members(key, ev.fork, ev.fork2, ev.join, true);
            cudaError_t e = cudaStreamEndCapture(key.origin, &graph);
            if (rc) {
                if (graph) cudaGraphDestroy(graph);
                return fail(rc);
            }
            if (e != cudaSuccess) return set_err(c0, DGV_ECUDA, std::string("group capture: ") + cudaGetErrorString(e));
            cudaGraphExec_t exec = nullptr;
            e = cudaGraphInstantiate(&exec, graph, 0);
            cudaGraphDestroy(graph);
            if (e != cudaSuccess)
                return set_err(c0, DGV_ECUDA, std::string("group instantiate: ") + cudaGetErrorString(e));
            GroupGraph &g2 = g_groups[key];
            if (g2.exec) cudaGraphExecDestroy(g2.exec);
            g2.exec = exec;
            g2.calls = 2;
            // capturing counted the launches once without running them
            g2.launches.clear();
            for (size_t i = 0; i < key.m.size(); i++) g2.launches.push_back(key.m[i].c->kt_all - before[i]);
            DGV_CUDA(c0, cudaGraphLaunch(exec, key.origin));
        }
    }
    if (c0->async) return DGV_OK;
    DGV_CUDA(c0, cudaStreamSynchronize(key.origin));
    for (const Member &mb : key.m) {
        int rc = check_errflag(mb.c);
        if (rc) return fail(rc);
    }
    return DGV_OK;
}
