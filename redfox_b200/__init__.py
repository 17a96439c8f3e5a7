"""redfox_b200: a B200-native (sm_100a) implementation of Red Fox's relational-algebra
kernel library.  The compute lives in librfx.so (C ABI in include/rfx/rfx.h); this
package is the host-side binding and the workload definitions."""
