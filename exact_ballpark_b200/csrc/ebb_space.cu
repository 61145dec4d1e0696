// SPDX-License-Identifier: MIT
// The space layer's tape on the device: one thread (or one warp) a world runs its K operations in order
// (ebb_space.cuh), over the state in either arrangement (interleaved [entry][world], or world-major). The parameter
// structs are __grid_constant__: the program reads its state's pointers through their addresses in the parameter
// space (uniform constant loads) rather than from a per-thread copy in local memory.
#include <cuda_runtime.h>

#include "../../include/ebb.h"
#include "ebb_space.cuh"

namespace ebb {
namespace space {

template <bool WM>
__global__ void __launch_bounds__(128, 6) tape_kernel(const __grid_constant__ EbbFlightState p,
                                                   const __grid_constant__ EbbSpaceState s,
                                                   const __grid_constant__ EbbSpaceTape t) {
    const int64_t w = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (w >= s.worlds) return;
    run_tape<WM>(&p, &s, &t, w);
}

// a warp a world: the world's index is the warp's, the lanes run its program together (ebb_space.cuh's World)
template <bool WM>
__global__ void __launch_bounds__(128, 12) tape_kernel_warp(const __grid_constant__ EbbFlightState p,
                                                         const __grid_constant__ EbbSpaceState s,
                                                         const __grid_constant__ EbbSpaceTape t) {
    __shared__ Coop scratch[4];
    const int64_t w = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (w >= s.worlds) return;                            // (the whole warp: w is the warp's)
    run_tape<WM, true>(&p, &s, &t, w, (int)(threadIdx.x & 31), &scratch[threadIdx.x >> 5]);
}

template <bool WM>
__global__ void __launch_bounds__(128) query_kernel(const __grid_constant__ EbbFlightState p,
                                                    const __grid_constant__ EbbSpaceState s,
                                                    const __grid_constant__ EbbSpaceQuery q) {
    const int64_t w = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (w >= s.worlds) return;
    run_query<WM>(&p, &s, &q, w);
}

}  // namespace space
}  // namespace ebb

extern "C" {

// the sizes and the block (checked first: a call with no worlds then does nothing), then every buffer
static int space_sizes(const EbbFlightState* park, const EbbSpaceState* s, int block) {
    if (park == nullptr || s == nullptr || block <= 0 || block > 128 || block % 32 != 0) return EBB_EINVAL;
    if (s->slots < 1 || s->slots > EBB_SPACE_MAX_SLOTS || s->boxes < 1 || s->dicts < 1 || s->entries < 1 ||
        s->sets < 1)
        return EBB_EINVAL;
    return 0;
}

static int space_buffers(const EbbFlightState* park, const EbbSpaceState* s) {
    if (s->rows == nullptr || s->level == nullptr || s->key == nullptr || s->mod == nullptr || s->active == nullptr ||
        s->bubble == nullptr || s->old_bubble == nullptr || s->seq == nullptr || s->in_park == nullptr ||
        s->keep_alive == nullptr || s->dead == nullptr || s->dropped == nullptr || s->box_level == nullptr ||
        s->box_key == nullptr || s->box_balls == nullptr || s->box_kids == nullptr || s->box_bubble == nullptr ||
        s->my_box == nullptr || s->my_top == nullptr || s->box_hash == nullptr || s->box_free == nullptr ||
        s->box_free_n == nullptr ||
        s->stack == nullptr || s->box_n == nullptr || s->free_boxes == nullptr || s->dict_bubble == nullptr ||
        s->dict_n == nullptr || s->entry_bubble == nullptr || s->entry_id == nullptr || s->entry_value == nullptr ||
        s->entry_n == nullptr || s->inter_bubble == nullptr || s->inter_id == nullptr || s->inter_n == nullptr ||
        s->keep_bubble == nullptr || s->keep_id == nullptr || s->keep_n == nullptr || s->bubble_id == nullptr ||
        s->seq_next == nullptr || s->flags == nullptr)
        return EBB_EINVAL;
    if (s->umap_cap < 1 || s->umap_cap > EBB_SPACE_MAX_SLOTS || s->events < 0 || s->srange == nullptr ||
        s->speriod == nullptr || s->selapsed == nullptr || s->ntf_range == nullptr || s->trk_range == nullptr ||
        s->trk == nullptr || s->cloaked == nullptr || s->sonly == nullptr || s->has_prox == nullptr ||
        s->ntf_in == nullptr || s->trk_in == nullptr || s->slist == nullptr || s->slen == nullptr ||
        s->sbkt == nullptr || s->pmap == nullptr || s->pn == nullptr || s->pbkt == nullptr || s->evn == nullptr ||
        s->rnd == nullptr || (s->events > 0 && s->ev == nullptr) || s->smask == nullptr || s->pmask == nullptr ||
        (s->lanes != 1 && s->lanes != 32) || s->pitch < 0 || s->pitch % 16 != 0 || s->box_parent == nullptr ||
        s->box_top == nullptr || s->box_home == nullptr || s->box_slot == nullptr || s->fbox == nullptr)
        return EBB_EINVAL;
    if (park->pos == nullptr || park->vel == nullptr || park->old_pos == nullptr || park->old_vel == nullptr ||
        park->ids == nullptr || park->radius == nullptr || park->max_vel == nullptr || park->agility == nullptr ||
        park->speed_fraction == nullptr || park->mass == nullptr || park->time_factor == nullptr ||
        park->free_ == nullptr || park->interactive == nullptr || park->mode == nullptr || park->goto_pt == nullptr ||
        park->follow_ptr == nullptr || park->follow_range == nullptr || park->massive == nullptr || park->sensor == nullptr)
        return EBB_EINVAL;
    return 0;
}

int ebb_space_tape(const EbbFlightState* park, const EbbSpaceState* s, const EbbSpaceTape* t, void* stream, int block) {
    if (t == nullptr || t->K < 0) return EBB_EINVAL;
    int rc = space_sizes(park, s, block);
    if (rc) return rc;
    if (s->worlds <= 0 || t->K == 0) return 0;
    rc = space_buffers(park, s);
    if (rc) return rc;
    if (t->code == nullptr || t->a == nullptr || t->b == nullptr) return EBB_EINVAL;
    const cudaStream_t st = (cudaStream_t)stream;
    if (s->lanes == 32) {
        const unsigned grid = (unsigned)((s->worlds * 32 + 127) / 128);
        if (s->pitch > 0)
            ebb::space::tape_kernel_warp<true><<<grid, 128, 0, st>>>(*park, *s, *t);
        else
            ebb::space::tape_kernel_warp<false><<<grid, 128, 0, st>>>(*park, *s, *t);
    } else {
        const unsigned grid = (unsigned)((s->worlds + block - 1) / block);
        if (s->pitch > 0)
            ebb::space::tape_kernel<true><<<grid, block, 0, st>>>(*park, *s, *t);
        else
            ebb::space::tape_kernel<false><<<grid, block, 0, st>>>(*park, *s, *t);
    }
    const cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? 0 : (int)e;
}

int ebb_space_query(const EbbFlightState* park, const EbbSpaceState* s, const EbbSpaceQuery* q, void* stream,
                    int block) {
    if (q == nullptr || q->kind < EBB_SPACE_Q_VISIBILITY || q->kind > EBB_SPACE_Q_NEARBY) return EBB_EINVAL;
    int rc = space_sizes(park, s, block);
    if (rc) return rc;
    if (s->worlds <= 0) return 0;
    rc = space_buffers(park, s);
    if (rc) return rc;
    if (q->a == nullptr || q->b == nullptr || q->f == nullptr || q->out == nullptr || q->outd == nullptr)
        return EBB_EINVAL;
    const unsigned grid = (unsigned)((s->worlds + block - 1) / block);
    if (s->pitch > 0)
        ebb::space::query_kernel<true><<<grid, block, 0, (cudaStream_t)stream>>>(*park, *s, *q);
    else
        ebb::space::query_kernel<false><<<grid, block, 0, (cudaStream_t)stream>>>(*park, *s, *q);
    const cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? 0 : (int)e;
}

}  // extern "C"

EBB_OP_COUNTER(ebb_count_ops_space)

#ifdef EBB_COUNT_OPS
// the counting build's tally of CheckSensor's paths: checks, re-filings skipped, filings unchanged
extern "C" int ebb_count_sensor_paths(unsigned long long* out, int reset) {
    cudaError_t e = cudaMemcpyFromSymbol(out, ebb::space::sensor_paths, sizeof(unsigned long long) * 3);
    if (e == cudaSuccess && reset) {
        const unsigned long long zero[3] = {};
        e = cudaMemcpyToSymbol(ebb::space::sensor_paths, zero, sizeof(zero));
    }
    return e == cudaSuccess ? 0 : (int)e;
}
#endif
