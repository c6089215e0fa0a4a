// Variants of the one-launch four-step kernel, part 2 (see pcx_fs_launch.cuh).
#include "pcx_fs_launch.cuh"

PCX_FS_PART(pcx_fs_part2) {
    PCX_FS_VARIANT(float, 9, 9, 1, 3)
    PCX_FS_VARIANT(float, 10, 8, 1, 3)
    PCX_FS_VARIANT(float, 8, 10, 1, 3)
    PCX_FS_VARIANT(float, 10, 9, 1, 2)
    PCX_FS_VARIANT(float, 10, 9, 1, 3)
    PCX_FS_VARIANT(float, 9, 10, 1, 2)
    return cudaErrorNotSupported;
}
