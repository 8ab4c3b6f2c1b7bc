// Run-time dispatch of the FP32-product walks on (n, real/complex).
#include "f32_impl.cuh"

namespace spb {
namespace dense {

int launch_walk_f32(const Problem& pb, int blocks, int threads, size_t smem, cudaStream_t s)
{
    switch (pb.n * 2 + (pb.comps == 2 ? 1 : 0)) {
    case 6: return launch_f32_n<3, 1>(pb, blocks, threads, smem, s);
    case 7: return launch_f32_n<3, 2>(pb, blocks, threads, smem, s);
    case 8: return launch_f32_n<4, 1>(pb, blocks, threads, smem, s);
    case 9: return launch_f32_n<4, 2>(pb, blocks, threads, smem, s);
    case 10: return launch_f32_n<5, 1>(pb, blocks, threads, smem, s);
    case 11: return launch_f32_n<5, 2>(pb, blocks, threads, smem, s);
    case 12: return launch_f32_n<6, 1>(pb, blocks, threads, smem, s);
    case 13: return launch_f32_n<6, 2>(pb, blocks, threads, smem, s);
    case 14: return launch_f32_n<7, 1>(pb, blocks, threads, smem, s);
    case 15: return launch_f32_n<7, 2>(pb, blocks, threads, smem, s);
    case 16: return launch_f32_n<8, 1>(pb, blocks, threads, smem, s);
    case 17: return launch_f32_n<8, 2>(pb, blocks, threads, smem, s);
    case 18: return launch_f32_n<9, 1>(pb, blocks, threads, smem, s);
    case 19: return launch_f32_n<9, 2>(pb, blocks, threads, smem, s);
    case 20: return launch_f32_n<10, 1>(pb, blocks, threads, smem, s);
    case 21: return launch_f32_n<10, 2>(pb, blocks, threads, smem, s);
    case 22: return launch_f32_n<11, 1>(pb, blocks, threads, smem, s);
    case 23: return launch_f32_n<11, 2>(pb, blocks, threads, smem, s);
    case 24: return launch_f32_n<12, 1>(pb, blocks, threads, smem, s);
    case 25: return launch_f32_n<12, 2>(pb, blocks, threads, smem, s);
    case 26: return launch_f32_n<13, 1>(pb, blocks, threads, smem, s);
    case 27: return launch_f32_n<13, 2>(pb, blocks, threads, smem, s);
    case 28: return launch_f32_n<14, 1>(pb, blocks, threads, smem, s);
    case 29: return launch_f32_n<14, 2>(pb, blocks, threads, smem, s);
    case 30: return launch_f32_n<15, 1>(pb, blocks, threads, smem, s);
    case 31: return launch_f32_n<15, 2>(pb, blocks, threads, smem, s);
    case 32: return launch_f32_n<16, 1>(pb, blocks, threads, smem, s);
    case 33: return launch_f32_n<16, 2>(pb, blocks, threads, smem, s);
    case 34: return launch_f32_n<17, 1>(pb, blocks, threads, smem, s);
    case 35: return launch_f32_n<17, 2>(pb, blocks, threads, smem, s);
    case 36: return launch_f32_n<18, 1>(pb, blocks, threads, smem, s);
    case 37: return launch_f32_n<18, 2>(pb, blocks, threads, smem, s);
    case 38: return launch_f32_n<19, 1>(pb, blocks, threads, smem, s);
    case 39: return launch_f32_n<19, 2>(pb, blocks, threads, smem, s);
    case 40: return launch_f32_n<20, 1>(pb, blocks, threads, smem, s);
    case 41: return launch_f32_n<20, 2>(pb, blocks, threads, smem, s);
    case 42: return launch_f32_n<21, 1>(pb, blocks, threads, smem, s);
    case 43: return launch_f32_n<21, 2>(pb, blocks, threads, smem, s);
    case 44: return launch_f32_n<22, 1>(pb, blocks, threads, smem, s);
    case 45: return launch_f32_n<22, 2>(pb, blocks, threads, smem, s);
    case 46: return launch_f32_n<23, 1>(pb, blocks, threads, smem, s);
    case 47: return launch_f32_n<23, 2>(pb, blocks, threads, smem, s);
    case 48: return launch_f32_n<24, 1>(pb, blocks, threads, smem, s);
    case 49: return launch_f32_n<24, 2>(pb, blocks, threads, smem, s);
    case 50: return launch_f32_n<25, 1>(pb, blocks, threads, smem, s);
    case 51: return launch_f32_n<25, 2>(pb, blocks, threads, smem, s);
    case 52: return launch_f32_n<26, 1>(pb, blocks, threads, smem, s);
    case 53: return launch_f32_n<26, 2>(pb, blocks, threads, smem, s);
    case 54: return launch_f32_n<27, 1>(pb, blocks, threads, smem, s);
    case 55: return launch_f32_n<27, 2>(pb, blocks, threads, smem, s);
    case 56: return launch_f32_n<28, 1>(pb, blocks, threads, smem, s);
    case 57: return launch_f32_n<28, 2>(pb, blocks, threads, smem, s);
    case 58: return launch_f32_n<29, 1>(pb, blocks, threads, smem, s);
    case 59: return launch_f32_n<29, 2>(pb, blocks, threads, smem, s);
    case 60: return launch_f32_n<30, 1>(pb, blocks, threads, smem, s);
    case 61: return launch_f32_n<30, 2>(pb, blocks, threads, smem, s);
    case 62: return launch_f32_n<31, 1>(pb, blocks, threads, smem, s);
    case 63: return launch_f32_n<31, 2>(pb, blocks, threads, smem, s);
    case 64: return launch_f32_n<32, 1>(pb, blocks, threads, smem, s);
    case 65: return launch_f32_n<32, 2>(pb, blocks, threads, smem, s);
    case 66: return launch_f32_n<33, 1>(pb, blocks, threads, smem, s);
    case 67: return launch_f32_n<33, 2>(pb, blocks, threads, smem, s);
    case 68: return launch_f32_n<34, 1>(pb, blocks, threads, smem, s);
    case 69: return launch_f32_n<34, 2>(pb, blocks, threads, smem, s);
    case 70: return launch_f32_n<35, 1>(pb, blocks, threads, smem, s);
    case 71: return launch_f32_n<35, 2>(pb, blocks, threads, smem, s);
    case 72: return launch_f32_n<36, 1>(pb, blocks, threads, smem, s);
    case 73: return launch_f32_n<36, 2>(pb, blocks, threads, smem, s);
    case 74: return launch_f32_n<37, 1>(pb, blocks, threads, smem, s);
    case 75: return launch_f32_n<37, 2>(pb, blocks, threads, smem, s);
    case 76: return launch_f32_n<38, 1>(pb, blocks, threads, smem, s);
    case 77: return launch_f32_n<38, 2>(pb, blocks, threads, smem, s);
    case 78: return launch_f32_n<39, 1>(pb, blocks, threads, smem, s);
    case 79: return launch_f32_n<39, 2>(pb, blocks, threads, smem, s);
    case 80: return launch_f32_n<40, 1>(pb, blocks, threads, smem, s);
    case 81: return launch_f32_n<40, 2>(pb, blocks, threads, smem, s);
    default:
        spb_set_error("FP32-product walk: n=%d outside 3..%d", pb.n, kMaxF32N);
        return SPB_ERR_INVALID;
    }
}

size_t walk_f32_smem_bytes(const Problem& pb, int threads) { return f32_smem_bytes(pb.n, pb.comps, pb.w, threads); }

int walk_f32_max_threads(int n, int comps) { return (comps == 1 && n <= 32) ? 512 : 256; }

}  // namespace dense
}  // namespace spb
