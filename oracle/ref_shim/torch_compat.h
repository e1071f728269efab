// torch_compat.h — force-included when compiling the reference extension against the
// torch in this image: the reference dispatches on tensor.type() (DeprecatedTypeProperties),
// which current AT_DISPATCH macros no longer convert to a ScalarType.  This adds that one
// conversion.  Used only by the reference build recipe (oracle/build_ref.py).
#pragma once
#include <ATen/ATen.h>
namespace detail {
inline at::ScalarType scalar_type(const at::DeprecatedTypeProperties& t) { return t.scalarType(); }
}
