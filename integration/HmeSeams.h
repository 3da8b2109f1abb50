// Installation of libhme behind the reference engine's seams (see HmeSeams.cpp).
#pragma once
#include <cstdint>

namespace hme_seams {

// Install the ring2k device LU table (ring2k::device::set_ops) and the device RREF hook
// (elim::set_device_rref_hook), both on GPU `device`.  Call once, before the first elimination.
void install(int device = 0);
// Remove both (the host code runs everywhere again).
void uninstall();

// Validation knobs (no value can change through them): a cap on the device LU's column window
// (0 = none; below the matrix width the tiled route runs), the tiled route's L-store budget in
// bytes (0 = HME_R2K_HOST_MB), the verify twin (1 on, 0 off, -1 HME_R2K_VERIFY), and the size
// floors of the device LU and the RREF hook in entries (0 = the environment's or 65536).
void set_r2k_max_cols(uint32_t cols);
void set_r2k_store_bytes(uint64_t bytes);
void set_r2k_verify(int on);
void set_min_entries(uint64_t r2k, uint64_t rref);

// Diagnostics: device LU sessions opened, RREF / rank-profile calls the hook served.
uint64_t r2k_sessions();
uint64_t rref_calls();

}  // namespace hme_seams
