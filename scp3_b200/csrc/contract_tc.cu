// Split-precision contraction (placeholder until the tcgen05 kernel lands).
#include "tc.h"

namespace scp3 {
namespace tc {

int create(Plan& p, int nb, int nm, int chunk_req, int sms)
{
    (void)p, (void)nb, (void)nm, (void)chunk_req, (void)sms;
    return fail(SCP3GPU_ERR_UNSUPPORTED, "BF16x3 contraction not built yet");
}
void destroy(Plan& p) { (void)p; }
int64_t pass_samples(const Plan& p, int64_t nvalid) { return (void)p, nvalid; }
int zero(Plan& p, cudaStream_t s) { return (void)p, (void)s, SCP3GPU_OK; }
int accumulate_pass(Plan&, const uint32_t*, int, int, const float*, const double*, int64_t, cudaStream_t,
                    std::vector<cudaEvent_t>*, std::vector<int>*)
{
    return fail(SCP3GPU_ERR_UNSUPPORTED, "BF16x3 contraction not built yet");
}
int unpack(Plan&, int, double, const double*, double, double*, int64_t, cudaStream_t)
{
    return fail(SCP3GPU_ERR_UNSUPPORTED, "BF16x3 contraction not built yet");
}

}  // namespace tc
}  // namespace scp3
