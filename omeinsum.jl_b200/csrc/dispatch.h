// Host-side einsum dispatch shared by the single-call API and the plan
// executor: labelled strided views, diagonal (repeated-label) views, label
// classification and mode sorting/merging.
#pragma once
#include <string>
#include "kernels.h"

struct ome_ctx {
  int device;
  int num_sms;
  char* ws;          // device workspace (plan intermediates, scratch)
  size_t ws_bytes;
  size_t ws_top;     // bump pointer; reset by every top-level call
  char* ovf;         // operand scratch of packed GEMMs that do not fit the workspace
  size_t ovf_bytes;  // (grown on demand outside stream capture; freed with the context)
};

namespace ome {

// A labelled strided tensor on the host side of the ABI.
struct HView {
  char* data = nullptr;
  int nd = 0;
  int64_t ext[MAXD];
  int64_t str[MAXD];
  int32_t lab[MAXD];
};

int set_err(int code, const char* fmt, ...);
int cuda_err(cudaError_t e, const char* what);

int view_from_tensor(const ome_tensor& t, HView& v, const char* what);
// Repeated labels -> one dimension with the summed stride (diagonal view).
int unique_view(const HView& v, HView& u);

void* ws_alloc(ome_ctx* c, size_t bytes);

// y <- sy*y + sx*f(xs) for labelled views (any number of inputs).
// loop_only forces the generic index kernel.
int einsum_views(ome_ctx* ctx, cudaStream_t s, ome_dtype dt, int nin, const HView* xs,
                 const HView& y, const Scalar& sx, const Scalar& sy, int prec, bool loop_only);

// Scalar helpers in the algebra of dt.
bool scalar_is_zero(ome_dtype dt, const Scalar& v);
bool scalar_is_one(ome_dtype dt, const Scalar& v);
Scalar scalar_one(ome_dtype dt);
Scalar scalar_zero(ome_dtype dt);
Scalar scalar_from(ome_dtype dt, const void* p);

// A plan's element type and number of inputs (plan.cu).
ome_dtype plan_dtype(const ome_plan* p);
int plan_ninputs(const ome_plan* p);

}  // namespace ome
