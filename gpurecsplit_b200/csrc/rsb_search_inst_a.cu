// Aggregation and leaf searches (stage kernels and the pipeline kernel) instantiated for leaf sizes 2..8 (the leaf sizes are
// split over several files so that they compile in parallel).
#include "rsb_pipeline_impl.cuh"

namespace rsb {
namespace search_impl {

template void run_aggr<2>(const SearchCtx &, int, const StageSchedule &, cudaStream_t);
template void run_partition<2>(const SearchCtx &, int, cudaStream_t);
template void run_leaves<2>(const SearchCtx &, int, const StageSchedule &, cudaStream_t);
template void run_aggr<3>(const SearchCtx &, int, const StageSchedule &, cudaStream_t);
template void run_partition<3>(const SearchCtx &, int, cudaStream_t);
template void run_leaves<3>(const SearchCtx &, int, const StageSchedule &, cudaStream_t);
template void run_aggr<4>(const SearchCtx &, int, const StageSchedule &, cudaStream_t);
template void run_partition<4>(const SearchCtx &, int, cudaStream_t);
template void run_leaves<4>(const SearchCtx &, int, const StageSchedule &, cudaStream_t);
template void run_aggr<5>(const SearchCtx &, int, const StageSchedule &, cudaStream_t);
template void run_partition<5>(const SearchCtx &, int, cudaStream_t);
template void run_leaves<5>(const SearchCtx &, int, const StageSchedule &, cudaStream_t);
template void run_aggr<6>(const SearchCtx &, int, const StageSchedule &, cudaStream_t);
template void run_partition<6>(const SearchCtx &, int, cudaStream_t);
template void run_leaves<6>(const SearchCtx &, int, const StageSchedule &, cudaStream_t);
template void run_aggr<7>(const SearchCtx &, int, const StageSchedule &, cudaStream_t);
template void run_partition<7>(const SearchCtx &, int, cudaStream_t);
template void run_leaves<7>(const SearchCtx &, int, const StageSchedule &, cudaStream_t);
template void run_aggr<8>(const SearchCtx &, int, const StageSchedule &, cudaStream_t);
template void run_partition<8>(const SearchCtx &, int, cudaStream_t);
template void run_leaves<8>(const SearchCtx &, int, const StageSchedule &, cudaStream_t);

template void run_pipeline<2>(const SearchCtx &, const PipeCtx &, const StageSchedule &, const StageSchedule &,
                                 cudaStream_t);
template void run_pipeline<3>(const SearchCtx &, const PipeCtx &, const StageSchedule &, const StageSchedule &,
                                 cudaStream_t);
template void run_pipeline<4>(const SearchCtx &, const PipeCtx &, const StageSchedule &, const StageSchedule &,
                                 cudaStream_t);
template void run_pipeline<5>(const SearchCtx &, const PipeCtx &, const StageSchedule &, const StageSchedule &,
                                 cudaStream_t);
template void run_pipeline<6>(const SearchCtx &, const PipeCtx &, const StageSchedule &, const StageSchedule &,
                                 cudaStream_t);
template void run_pipeline<7>(const SearchCtx &, const PipeCtx &, const StageSchedule &, const StageSchedule &,
                                 cudaStream_t);
template void run_pipeline<8>(const SearchCtx &, const PipeCtx &, const StageSchedule &, const StageSchedule &,
                                 cudaStream_t);

}  // namespace search_impl
}  // namespace rsb
