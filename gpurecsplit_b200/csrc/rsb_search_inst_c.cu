// Aggregation and leaf searches (stage kernels and the pipeline kernel) instantiated for leaf sizes 15..19 (the leaf sizes are
// split over several files so that they compile in parallel).
#include "rsb_pipeline_impl.cuh"

namespace rsb {
namespace search_impl {

template void run_aggr<15>(const SearchCtx &, int, const StageSchedule &, cudaStream_t);
template void run_partition<15>(const SearchCtx &, int, cudaStream_t);
template void run_leaves<15>(const SearchCtx &, int, const StageSchedule &, cudaStream_t);
template void run_aggr<16>(const SearchCtx &, int, const StageSchedule &, cudaStream_t);
template void run_partition<16>(const SearchCtx &, int, cudaStream_t);
template void run_leaves<16>(const SearchCtx &, int, const StageSchedule &, cudaStream_t);
template void run_aggr<17>(const SearchCtx &, int, const StageSchedule &, cudaStream_t);
template void run_partition<17>(const SearchCtx &, int, cudaStream_t);
template void run_leaves<17>(const SearchCtx &, int, const StageSchedule &, cudaStream_t);
template void run_aggr<18>(const SearchCtx &, int, const StageSchedule &, cudaStream_t);
template void run_partition<18>(const SearchCtx &, int, cudaStream_t);
template void run_leaves<18>(const SearchCtx &, int, const StageSchedule &, cudaStream_t);
template void run_aggr<19>(const SearchCtx &, int, const StageSchedule &, cudaStream_t);
template void run_partition<19>(const SearchCtx &, int, cudaStream_t);
template void run_leaves<19>(const SearchCtx &, int, const StageSchedule &, cudaStream_t);

template void run_pipeline<15>(const SearchCtx &, const PipeCtx &, const StageSchedule &, const StageSchedule &,
                                 cudaStream_t);
template void run_pipeline<16>(const SearchCtx &, const PipeCtx &, const StageSchedule &, const StageSchedule &,
                                 cudaStream_t);
template void run_pipeline<17>(const SearchCtx &, const PipeCtx &, const StageSchedule &, const StageSchedule &,
                                 cudaStream_t);
template void run_pipeline<18>(const SearchCtx &, const PipeCtx &, const StageSchedule &, const StageSchedule &,
                                 cudaStream_t);
template void run_pipeline<19>(const SearchCtx &, const PipeCtx &, const StageSchedule &, const StageSchedule &,
                                 cudaStream_t);

}  // namespace search_impl
}  // namespace rsb
