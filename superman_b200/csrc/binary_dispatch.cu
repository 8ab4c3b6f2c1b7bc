// Run-time dispatch of walk_binary on (limbs, n).
#include "binary_launch.cuh"

namespace spb {
namespace binary {

int launch_binary(const Problem& pb, int blocks, int threads, size_t smem, cudaStream_t s)
{
    switch (pb.limbs * 100 + pb.n) {
    case 401: return launch_bin_n<1, 4>(pb, blocks, threads, smem, s);
    case 402: return launch_bin_n<2, 4>(pb, blocks, threads, smem, s);
    case 403: return launch_bin_n<3, 4>(pb, blocks, threads, smem, s);
    case 404: return launch_bin_n<4, 4>(pb, blocks, threads, smem, s);
    case 405: return launch_bin_n<5, 4>(pb, blocks, threads, smem, s);
    case 406: return launch_bin_n<6, 4>(pb, blocks, threads, smem, s);
    case 407: return launch_bin_n<7, 4>(pb, blocks, threads, smem, s);
    case 408: return launch_bin_n<8, 4>(pb, blocks, threads, smem, s);
    case 409: return launch_bin_n<9, 4>(pb, blocks, threads, smem, s);
    case 410: return launch_bin_n<10, 4>(pb, blocks, threads, smem, s);
    case 411: return launch_bin_n<11, 4>(pb, blocks, threads, smem, s);
    case 412: return launch_bin_n<12, 4>(pb, blocks, threads, smem, s);
    case 413: return launch_bin_n<13, 4>(pb, blocks, threads, smem, s);
    case 414: return launch_bin_n<14, 4>(pb, blocks, threads, smem, s);
    case 415: return launch_bin_n<15, 4>(pb, blocks, threads, smem, s);
    case 416: return launch_bin_n<16, 4>(pb, blocks, threads, smem, s);
    case 417: return launch_bin_n<17, 4>(pb, blocks, threads, smem, s);
    case 418: return launch_bin_n<18, 4>(pb, blocks, threads, smem, s);
    case 419: return launch_bin_n<19, 4>(pb, blocks, threads, smem, s);
    case 420: return launch_bin_n<20, 4>(pb, blocks, threads, smem, s);
    case 421: return launch_bin_n<21, 4>(pb, blocks, threads, smem, s);
    case 422: return launch_bin_n<22, 4>(pb, blocks, threads, smem, s);
    case 423: return launch_bin_n<23, 4>(pb, blocks, threads, smem, s);
    case 424: return launch_bin_n<24, 4>(pb, blocks, threads, smem, s);
    case 425: return launch_bin_n<25, 4>(pb, blocks, threads, smem, s);
    case 426: return launch_bin_n<26, 4>(pb, blocks, threads, smem, s);
    case 427: return launch_bin_n<27, 4>(pb, blocks, threads, smem, s);
    case 428: return launch_bin_n<28, 4>(pb, blocks, threads, smem, s);
    case 429: return launch_bin_n<29, 4>(pb, blocks, threads, smem, s);
    case 430: return launch_bin_n<30, 4>(pb, blocks, threads, smem, s);
    case 431: return launch_bin_n<31, 4>(pb, blocks, threads, smem, s);
    case 432: return launch_bin_n<32, 4>(pb, blocks, threads, smem, s);
    case 433: return launch_bin_n<33, 4>(pb, blocks, threads, smem, s);
    case 434: return launch_bin_n<34, 4>(pb, blocks, threads, smem, s);
    case 435: return launch_bin_n<35, 4>(pb, blocks, threads, smem, s);
    case 436: return launch_bin_n<36, 4>(pb, blocks, threads, smem, s);
    case 437: return launch_bin_n<37, 4>(pb, blocks, threads, smem, s);
    case 438: return launch_bin_n<38, 4>(pb, blocks, threads, smem, s);
    case 439: return launch_bin_n<39, 4>(pb, blocks, threads, smem, s);
    case 440: return launch_bin_n<40, 4>(pb, blocks, threads, smem, s);
    case 441: return launch_bin_n<41, 4>(pb, blocks, threads, smem, s);
    case 442: return launch_bin_n<42, 4>(pb, blocks, threads, smem, s);
    case 443: return launch_bin_n<43, 4>(pb, blocks, threads, smem, s);
    case 444: return launch_bin_n<44, 4>(pb, blocks, threads, smem, s);
    case 445: return launch_bin_n<45, 4>(pb, blocks, threads, smem, s);
    case 446: return launch_bin_n<46, 4>(pb, blocks, threads, smem, s);
    case 447: return launch_bin_n<47, 4>(pb, blocks, threads, smem, s);
    case 448: return launch_bin_n<48, 4>(pb, blocks, threads, smem, s);
    case 449: return launch_bin_n<49, 4>(pb, blocks, threads, smem, s);
    case 450: return launch_bin_n<50, 4>(pb, blocks, threads, smem, s);
    case 451: return launch_bin_n<51, 4>(pb, blocks, threads, smem, s);
    case 452: return launch_bin_n<52, 4>(pb, blocks, threads, smem, s);
    case 453: return launch_bin_n<53, 4>(pb, blocks, threads, smem, s);
    case 454: return launch_bin_n<54, 4>(pb, blocks, threads, smem, s);
    case 455: return launch_bin_n<55, 4>(pb, blocks, threads, smem, s);
    case 456: return launch_bin_n<56, 4>(pb, blocks, threads, smem, s);
    case 457: return launch_bin_n<57, 4>(pb, blocks, threads, smem, s);
    case 458: return launch_bin_n<58, 4>(pb, blocks, threads, smem, s);
    case 459: return launch_bin_n<59, 4>(pb, blocks, threads, smem, s);
    case 460: return launch_bin_n<60, 4>(pb, blocks, threads, smem, s);
    case 461: return launch_bin_n<61, 4>(pb, blocks, threads, smem, s);
    case 462: return launch_bin_n<62, 4>(pb, blocks, threads, smem, s);
    case 463: return launch_bin_n<63, 4>(pb, blocks, threads, smem, s);
    case 634: return launch_bin_n<34, 6>(pb, blocks, threads, smem, s);
    case 635: return launch_bin_n<35, 6>(pb, blocks, threads, smem, s);
    case 636: return launch_bin_n<36, 6>(pb, blocks, threads, smem, s);
    case 637: return launch_bin_n<37, 6>(pb, blocks, threads, smem, s);
    case 638: return launch_bin_n<38, 6>(pb, blocks, threads, smem, s);
    case 639: return launch_bin_n<39, 6>(pb, blocks, threads, smem, s);
    case 640: return launch_bin_n<40, 6>(pb, blocks, threads, smem, s);
    case 641: return launch_bin_n<41, 6>(pb, blocks, threads, smem, s);
    case 642: return launch_bin_n<42, 6>(pb, blocks, threads, smem, s);
    case 643: return launch_bin_n<43, 6>(pb, blocks, threads, smem, s);
    case 644: return launch_bin_n<44, 6>(pb, blocks, threads, smem, s);
    case 645: return launch_bin_n<45, 6>(pb, blocks, threads, smem, s);
    case 646: return launch_bin_n<46, 6>(pb, blocks, threads, smem, s);
    case 647: return launch_bin_n<47, 6>(pb, blocks, threads, smem, s);
    case 648: return launch_bin_n<48, 6>(pb, blocks, threads, smem, s);
    case 649: return launch_bin_n<49, 6>(pb, blocks, threads, smem, s);
    case 650: return launch_bin_n<50, 6>(pb, blocks, threads, smem, s);
    case 651: return launch_bin_n<51, 6>(pb, blocks, threads, smem, s);
    case 652: return launch_bin_n<52, 6>(pb, blocks, threads, smem, s);
    case 653: return launch_bin_n<53, 6>(pb, blocks, threads, smem, s);
    case 654: return launch_bin_n<54, 6>(pb, blocks, threads, smem, s);
    case 655: return launch_bin_n<55, 6>(pb, blocks, threads, smem, s);
    case 656: return launch_bin_n<56, 6>(pb, blocks, threads, smem, s);
    case 657: return launch_bin_n<57, 6>(pb, blocks, threads, smem, s);
    case 658: return launch_bin_n<58, 6>(pb, blocks, threads, smem, s);
    case 659: return launch_bin_n<59, 6>(pb, blocks, threads, smem, s);
    case 660: return launch_bin_n<60, 6>(pb, blocks, threads, smem, s);
    case 661: return launch_bin_n<61, 6>(pb, blocks, threads, smem, s);
    case 662: return launch_bin_n<62, 6>(pb, blocks, threads, smem, s);
    case 663: return launch_bin_n<63, 6>(pb, blocks, threads, smem, s);
    case 1046: return launch_bin_n<46, 10>(pb, blocks, threads, smem, s);
    case 1047: return launch_bin_n<47, 10>(pb, blocks, threads, smem, s);
    case 1048: return launch_bin_n<48, 10>(pb, blocks, threads, smem, s);
    case 1049: return launch_bin_n<49, 10>(pb, blocks, threads, smem, s);
    case 1050: return launch_bin_n<50, 10>(pb, blocks, threads, smem, s);
    case 1051: return launch_bin_n<51, 10>(pb, blocks, threads, smem, s);
    case 1052: return launch_bin_n<52, 10>(pb, blocks, threads, smem, s);
    case 1053: return launch_bin_n<53, 10>(pb, blocks, threads, smem, s);
    case 1054: return launch_bin_n<54, 10>(pb, blocks, threads, smem, s);
    case 1055: return launch_bin_n<55, 10>(pb, blocks, threads, smem, s);
    case 1056: return launch_bin_n<56, 10>(pb, blocks, threads, smem, s);
    case 1057: return launch_bin_n<57, 10>(pb, blocks, threads, smem, s);
    case 1058: return launch_bin_n<58, 10>(pb, blocks, threads, smem, s);
    case 1059: return launch_bin_n<59, 10>(pb, blocks, threads, smem, s);
    case 1060: return launch_bin_n<60, 10>(pb, blocks, threads, smem, s);
    case 1061: return launch_bin_n<61, 10>(pb, blocks, threads, smem, s);
    case 1062: return launch_bin_n<62, 10>(pb, blocks, threads, smem, s);
    case 1063: return launch_bin_n<63, 10>(pb, blocks, threads, smem, s);
    default:
        spb_set_error("binary walk: no kernel for n=%d with %d limbs", pb.n, pb.limbs);
        return SPB_ERR_INVALID;
    }
}

}  // namespace binary
}  // namespace spb
