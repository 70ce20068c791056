// Stage launchers of the persistent seed searches (aggregation levels, their partitions and
// the leaves), defined in rsb_search_impl.cuh and instantiated per leaf size in
// rsb_search_inst_*.cu; rsb_search.cu dispatches to them by leaf size.
#pragma once

#include "rsb_kernels.cuh"

namespace rsb {
namespace search_impl {

template <int LEAF>
void run_aggr(const SearchCtx &c, int stage, const StageSchedule &s, cudaStream_t st);
template <int LEAF>
void run_partition(const SearchCtx &c, int stage, cudaStream_t st);
template <int LEAF>
void run_leaves(const SearchCtx &c, int stage, const StageSchedule &s, cudaStream_t st);
template <int LEAF>
void run_pipeline(const SearchCtx &c, const PipeCtx &p, const StageSchedule &aggr, const StageSchedule &leaf,
                  cudaStream_t st);

}  // namespace search_impl
}  // namespace rsb
