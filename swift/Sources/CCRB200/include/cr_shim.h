/* The library's C ABI for the Swift module map (unverified: no Swift
 * toolchain was available where this was written). */
#include "../../../../include/cr/cr.h"
