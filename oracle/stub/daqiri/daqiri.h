/* Minimal stand-in for the DAQIRI API surface that the reference's
 * src/rx_host_corr.cu uses (:128-131, :185-186, :245), so that file can be
 * compiled here to reach its kernels.  TEST INFRASTRUCTURE ONLY: nothing in
 * it moves packets; every call reports failure. */
#pragma once
#include <cstddef>
#include <cstdint>
namespace daqiri {
enum class Status { SUCCESS = 0, FAILURE = 1 };
struct BurstParams {
    int unused;
};
inline Status daqiri_init(const char*) { return Status::FAILURE; }
inline int get_port_id(const char*) { return -1; }
inline Status get_rx_burst(BurstParams** b, int, int) {
    *b = nullptr;
    return Status::FAILURE;
}
inline int64_t get_num_packets(BurstParams*) { return 0; }
inline void* get_packet_ptr(BurstParams*, int) { return nullptr; }
inline void free_all_packets_and_burst_rx(BurstParams*) {}
inline void print_stats() {}
inline void shutdown() {}
}  // namespace daqiri
