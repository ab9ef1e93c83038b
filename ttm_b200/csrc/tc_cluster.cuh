// Thread-block-cluster helpers of the SM-pair tensor-core kernels (tc_pair.cu, tc_pair8.cu):
// cluster coordinates, shared-memory addresses in the peer CTA, cross-CTA mbarrier arrivals,
// the cluster barrier, the multicast tcgen05.commit and 32-lane tensor-memory stores.
#pragma once

#include <cstdint>

#include "tc_ptx.cuh"

namespace tlibttm {
namespace {

__device__ __forceinline__ uint32_t cluster_rank()
{
    uint32_t r;
    asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
    return r;
}
__device__ __forceinline__ uint32_t cluster_index()
{
    uint32_t r;
    asm volatile("mov.u32 %0, %%clusterid.x;" : "=r"(r));
    return r;
}
__device__ __forceinline__ uint32_t cluster_count()
{
    uint32_t r;
    asm volatile("mov.u32 %0, %%nclusterid.x;" : "=r"(r));
    return r;
}
// Address of the same shared-memory variable in CTA `rank` of the cluster.
__device__ __forceinline__ uint32_t peer_addr(uint32_t saddr, uint32_t rank)
{
    uint32_t r;
    asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(r) : "r"(saddr), "r"(rank));
    return r;
}
// Arrive on a barrier of another CTA of the cluster (default semantics: release at CTA scope).
// What the arrive publishes is either shared memory the MMA reads, after fence.proxy.async, or
// tensor memory this CTA has finished loading, after tcgen05.fence::before_thread_sync; neither
// needs the thread's earlier global stores to be visible, which a cluster-scope release would
// wait for.
__device__ __forceinline__ void mbar_arrive_remote(uint32_t cluster_addr)
{
    asm volatile("mbarrier.arrive.shared::cluster.b64 _, [%0];" ::"r"(cluster_addr) : "memory");
}
__device__ __forceinline__ void cluster_sync_all()
{
    asm volatile("barrier.cluster.arrive.release.aligned;\n\tbarrier.cluster.wait.acquire.aligned;" ::: "memory");
}
// Arrive on the barrier at this offset in every CTA of `mask` once the MMAs issued so far are
// done (whole warp; one elected lane commits).
__device__ __forceinline__ void commit_pair(uint64_t* bar, uint16_t mask)
{
    asm volatile("{\n .reg .pred e;\n elect.sync _|e, 0xffffffff;\n"
                 " @e tcgen05.commit.cta_group::2.mbarrier::arrive::one.shared::cluster.multicast::cluster.b64 [%0], %1;\n}\n"
                 ::"r"(su32(bar)), "h"(mask)
                 : "memory");
}
__device__ __forceinline__ void tmem_st8(uint32_t taddr, const uint32_t (&r)[8])
{
    asm volatile("tcgen05.st.sync.aligned.32x32b.x8.b32 [%0], {%1, %2, %3, %4, %5, %6, %7, %8};"
                 ::"r"(taddr), "r"(r[0]), "r"(r[1]), "r"(r[2]), "r"(r[3]), "r"(r[4]), "r"(r[5]), "r"(r[6]), "r"(r[7])
                 : "memory");
}
// Arrive on a barrier of a CTA of the cluster with release at cluster scope: the arriving
// thread's earlier shared-memory stores (its own CTA's or, through st_cluster, the peer's) are
// visible to a thread whose wait on that phase has acquire at cluster scope.
__device__ __forceinline__ void mbar_arrive_remote_release_cluster(uint32_t cluster_addr)
{
    asm volatile("mbarrier.arrive.release.cluster.shared::cluster.b64 _, [%0];" ::"r"(cluster_addr) : "memory");
}
// 32-bit store to shared memory of a CTA of the cluster (address from peer_addr).
__device__ __forceinline__ void st_cluster_u32(uint32_t cluster_addr, uint32_t v)
{
    asm volatile("st.shared::cluster.u32 [%0], %1;" ::"r"(cluster_addr), "r"(v) : "memory");
}
__device__ __forceinline__ void fence_acq_rel_cluster() { asm volatile("fence.acq_rel.cluster;" ::: "memory"); }
// Bounded wait with acquire at cluster scope (pairs with mbar_arrive_remote_release_cluster).
__device__ __forceinline__ bool mbar_wait_cluster(uint64_t* bar, uint32_t phase, volatile int* abort_flag,
                                                  unsigned long long limit_ns)
{
    const unsigned long long t0 = gtimer();
    while (true) {
        uint32_t ok;
        asm volatile(
            "{\n .reg .pred p;\n mbarrier.try_wait.parity.acquire.cluster.shared::cta.b64 p, [%1], %2, %3;\n"
            " selp.u32 %0, 1, 0, p;\n}\n"
            : "=r"(ok)
            : "r"(su32(bar)), "r"(phase), "r"(kSleepHintNs)
            : "memory");
        if (ok) return true;
        if (*abort_flag) return false;
        if (gtimer() - t0 > limit_ns) {
            *abort_flag = 1;
            return false;
        }
    }
}

}  // namespace
}  // namespace tlibttm
