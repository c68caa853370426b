/* Forced-include shim for compiling the reference's GPU kernels (src/kernelInvocations.cu)
 * for sm_100a -- TEST INFRASTRUCTURE.  The reference was written for sm_30 and uses the warp
 * votes and shuffles without a member mask, which CUDA removed for sm_70 and later; these
 * map them onto the _sync forms over the active lanes.  The reference's traversal keeps
 * its warps converged (every branch is taken by __any of the warp), so the active mask is
 * the whole warp wherever they are used. */
#pragma once
#define __any(p) __any_sync(__activemask(), (p))
#define __all(p) __all_sync(__activemask(), (p))
#define __shfl_xor(v, m) __shfl_xor_sync(__activemask(), (v), (m))
#define __shfl(v, l) __shfl_sync(__activemask(), (v), (l))
