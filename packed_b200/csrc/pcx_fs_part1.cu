// Variants of the one-launch four-step kernel, part 1 (see pcx_fs_launch.cuh).
#include "pcx_fs_launch.cuh"

PCX_FS_PART(pcx_fs_part1) {
    PCX_FS_VARIANT(float, 8, 8, 1, 3)
    PCX_FS_VARIANT(float, 9, 8, 2, 3)
    PCX_FS_VARIANT(float, 8, 9, 2, 3)
    PCX_FS_VARIANT(float, 9, 8, 1, 3)
    PCX_FS_VARIANT(float, 10, 7, 1, 3)
    PCX_FS_VARIANT(float, 9, 9, 2, 3)
    return cudaErrorNotSupported;
}
