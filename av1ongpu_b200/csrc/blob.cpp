/*
 * blob.cpp - the serialized FrameSyntax ("blob", flat_syntax.hpp) at the C
 * ABI: a view into a blob without copying, and its patchable reference slot
 * list.
 */
#include "../../include/av1b.h"
#include "flat_syntax.hpp"

extern "C" {

int av1b_syntax_view(const uint8_t* blob, size_t len, av1b_frame_syntax* out) {
  if (!out) return AV1B_ERR_ARG;
  return av1b::view_blob(blob, len, out) ? AV1B_OK : AV1B_ERR_ARG;
}

int av1b_blob_set_refs(uint8_t* blob, size_t len, const int32_t* slots, int n) {
  return av1b::blob_set_refs(blob, len, slots, n) ? AV1B_OK : AV1B_ERR_ARG;
}

int av1b_blob_get_refs(const uint8_t* blob, size_t len, int32_t* slots, int max_n) {
  av1b_frame_syntax v;
  if (!av1b::view_blob(blob, len, &v)) return AV1B_ERR_ARG;
  const int n = static_cast<int>(v.n_reference_slots);
  for (int i = 0; i < n && i < max_n; ++i) slots[i] = v.reference_slots[i];
  return n;
}

}  // extern "C"
