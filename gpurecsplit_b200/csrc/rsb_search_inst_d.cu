// Aggregation and leaf searches (stage kernels and the pipeline kernel) instantiated for leaf sizes 20..24 (the leaf sizes are
// split over several files so that they compile in parallel).
#include "rsb_pipeline_impl.cuh"

namespace rsb {
namespace search_impl {

template void run_aggr<20>(const SearchCtx &, int, const StageSchedule &, cudaStream_t);
template void run_partition<20>(const SearchCtx &, int, cudaStream_t);
template void run_leaves<20>(const SearchCtx &, int, const StageSchedule &, cudaStream_t);
template void run_aggr<21>(const SearchCtx &, int, const StageSchedule &, cudaStream_t);
template void run_partition<21>(const SearchCtx &, int, cudaStream_t);
template void run_leaves<21>(const SearchCtx &, int, const StageSchedule &, cudaStream_t);
template void run_aggr<22>(const SearchCtx &, int, const StageSchedule &, cudaStream_t);
template void run_partition<22>(const SearchCtx &, int, cudaStream_t);
template void run_leaves<22>(const SearchCtx &, int, const StageSchedule &, cudaStream_t);
template void run_aggr<23>(const SearchCtx &, int, const StageSchedule &, cudaStream_t);
template void run_partition<23>(const SearchCtx &, int, cudaStream_t);
template void run_leaves<23>(const SearchCtx &, int, const StageSchedule &, cudaStream_t);
template void run_aggr<24>(const SearchCtx &, int, const StageSchedule &, cudaStream_t);
template void run_partition<24>(const SearchCtx &, int, cudaStream_t);
template void run_leaves<24>(const SearchCtx &, int, const StageSchedule &, cudaStream_t);

template void run_pipeline<20>(const SearchCtx &, const PipeCtx &, const StageSchedule &, const StageSchedule &,
                                 cudaStream_t);
template void run_pipeline<21>(const SearchCtx &, const PipeCtx &, const StageSchedule &, const StageSchedule &,
                                 cudaStream_t);
template void run_pipeline<22>(const SearchCtx &, const PipeCtx &, const StageSchedule &, const StageSchedule &,
                                 cudaStream_t);
template void run_pipeline<23>(const SearchCtx &, const PipeCtx &, const StageSchedule &, const StageSchedule &,
                                 cudaStream_t);
template void run_pipeline<24>(const SearchCtx &, const PipeCtx &, const StageSchedule &, const StageSchedule &,
                                 cudaStream_t);

}  // namespace search_impl
}  // namespace rsb
