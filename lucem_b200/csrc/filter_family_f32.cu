// filter_family_f32.cu -- the Gaussian-family tile kernels for float input
// (filter_family.cuh), in a translation unit of their own.
#include "filter_family.cuh"

namespace lucem {
namespace famk {

int planes_f32(const FamParams &p, void *stream) { return planes_t<float>(p, stream); }

int batch_f32(const FamParams &p, const FamImage *items_dev, int32_t n_items, int32_t n_tiles, void *stream) {
    return batch_t<float>(p, items_dev, n_items, n_tiles, stream);
}

int work_f32(const FamParams &p, const FamWork *work_dev, int32_t n_work, int32_t n_tiles_total, int32_t tile_base,
               int32_t *counter_dev, int32_t persistent_ctas, void *stream) {
    return work_t<float>(p, work_dev, n_work, n_tiles_total, tile_base, counter_dev, persistent_ctas, stream);
}

}  // namespace famk
}  // namespace lucem
