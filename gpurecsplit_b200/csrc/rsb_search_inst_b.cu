// Aggregation and leaf searches (stage kernels and the pipeline kernel) instantiated for leaf sizes 9..14 (the leaf sizes are
// split over several files so that they compile in parallel).
#include "rsb_pipeline_impl.cuh"

namespace rsb {
namespace search_impl {

template void run_aggr<9>(const SearchCtx &, int, const StageSchedule &, cudaStream_t);
template void run_partition<9>(const SearchCtx &, int, cudaStream_t);
template void run_leaves<9>(const SearchCtx &, int, const StageSchedule &, cudaStream_t);
template void run_aggr<10>(const SearchCtx &, int, const StageSchedule &, cudaStream_t);
template void run_partition<10>(const SearchCtx &, int, cudaStream_t);
template void run_leaves<10>(const SearchCtx &, int, const StageSchedule &, cudaStream_t);
template void run_aggr<11>(const SearchCtx &, int, const StageSchedule &, cudaStream_t);
template void run_partition<11>(const SearchCtx &, int, cudaStream_t);
template void run_leaves<11>(const SearchCtx &, int, const StageSchedule &, cudaStream_t);
template void run_aggr<12>(const SearchCtx &, int, const StageSchedule &, cudaStream_t);
template void run_partition<12>(const SearchCtx &, int, cudaStream_t);
template void run_leaves<12>(const SearchCtx &, int, const StageSchedule &, cudaStream_t);
template void run_aggr<13>(const SearchCtx &, int, const StageSchedule &, cudaStream_t);
template void run_partition<13>(const SearchCtx &, int, cudaStream_t);
template void run_leaves<13>(const SearchCtx &, int, const StageSchedule &, cudaStream_t);
template void run_aggr<14>(const SearchCtx &, int, const StageSchedule &, cudaStream_t);
template void run_partition<14>(const SearchCtx &, int, cudaStream_t);
template void run_leaves<14>(const SearchCtx &, int, const StageSchedule &, cudaStream_t);

template void run_pipeline<9>(const SearchCtx &, const PipeCtx &, const StageSchedule &, const StageSchedule &,
                                 cudaStream_t);
template void run_pipeline<10>(const SearchCtx &, const PipeCtx &, const StageSchedule &, const StageSchedule &,
                                 cudaStream_t);
template void run_pipeline<11>(const SearchCtx &, const PipeCtx &, const StageSchedule &, const StageSchedule &,
                                 cudaStream_t);
template void run_pipeline<12>(const SearchCtx &, const PipeCtx &, const StageSchedule &, const StageSchedule &,
                                 cudaStream_t);
template void run_pipeline<13>(const SearchCtx &, const PipeCtx &, const StageSchedule &, const StageSchedule &,
                                 cudaStream_t);
template void run_pipeline<14>(const SearchCtx &, const PipeCtx &, const StageSchedule &, const StageSchedule &,
                                 cudaStream_t);

}  // namespace search_impl
}  // namespace rsb
