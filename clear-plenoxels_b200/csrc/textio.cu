// textio.cu -- the reference's text file formats, for interop with its outputs.
//
// Grid checkpoints (objectScene::saveSelf / initFromFile, SVRF/SceneUtils.cu:1246-1300,
// 703-790; saveChannelSHs / loadChannelSHs :1209-1243, 659-701): one text file per array,
// rows of "%.6lf " values ending in "\n" (saveFloaters2File, Utils.cu:648-675), read back with
// fscanf("%f ") (readFloatersFromFile, :624-646); byte grids as "%d " rows (saveUchar2File /
// saveInt2File, :575-622).  Images (Image::initSelfFromFile, ImageUtils.cu:84-128): "%d " byte
// grids per channel and a mask whose nonzero pixels bound the mask-area rectangle (readMask,
// Utils.cu:508-552; processMasksInfo, ImageUtils.cu:130-146).  Host code: the grid's arrays
// move through the planar upload and download calls.
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "cpx_internal.cuh"

using namespace cpx;

namespace {

std::string join(const char* dir, const char* name) { return std::string(dir) + "/" + name; }

bool write_floats(const std::string& path, const float* a, int64_t rows, int64_t cols)
{
    FILE* f = std::fopen(path.c_str(), "w");
    if (!f) return false;
    for (int64_t r = 0; r < rows; r++) {
        for (int64_t c = 0; c < cols; c++) std::fprintf(f, "%.6lf ", (double)a[r * cols + c]);
        std::fprintf(f, "\n");
    }
    return std::fclose(f) == 0;
}

template <typename T>
bool write_ints(const std::string& path, const T* a, int64_t rows, int64_t cols)
{
    FILE* f = std::fopen(path.c_str(), "w");
    if (!f) return false;
    for (int64_t r = 0; r < rows; r++) {
        for (int64_t c = 0; c < cols; c++) std::fprintf(f, "%d ", (int)a[r * cols + c]);
        std::fprintf(f, "\n");
    }
    return std::fclose(f) == 0;
}

bool read_floats(const std::string& path, float* a, int64_t n)
{
    FILE* f = std::fopen(path.c_str(), "r");
    if (!f) return false;
    bool ok = true;
    for (int64_t i = 0; i < n && ok; i++) ok = std::fscanf(f, "%f ", a + i) == 1;
    std::fclose(f);
    return ok;
}

bool read_bytes(const std::string& path, uint8_t* a, int64_t n)
{
    FILE* f = std::fopen(path.c_str(), "r");
    if (!f) return false;
    bool ok = true;
    for (int64_t i = 0; i < n && ok; i++) {
        int v = 0;
        ok = std::fscanf(f, "%d ", &v) == 1;
        a[i] = (uint8_t)v;
    }
    std::fclose(f);
    return ok;
}

bool read_u32(const std::string& path, uint32_t* a, int64_t n)
{
    FILE* f = std::fopen(path.c_str(), "r");
    if (!f) return false;
    bool ok = true;
    for (int64_t i = 0; i < n && ok; i++) {
        int v = 0;
        ok = std::fscanf(f, "%d ", &v) == 1;
        a[i] = (uint32_t)v;
    }
    std::fclose(f);
    return ok;
}

cpx_status io_error(const std::string& path, const char* what)
{
    set_error("%s %s failed", what, path.c_str());
    return CPX_ERR_INVALID_ARGUMENT;
}

}  // namespace

extern "C" {

cpx_status cpx_grid_save_text(const cpx_grid* g, const char* dir, int band, int density_only, int hierarchy_mode)
{
    if (!g || !dir) {
        set_error("null argument");
        return CPX_ERR_INVALID_ARGUMENT;
    }
    const int files_sh = (band + 1) * (band + 1);
    if (band < 0 || files_sh > g->sh_dim) {
        set_error("band %d needs %d coefficients, the grid holds %d", band, files_sh, g->sh_dim);
        return CPX_ERR_INVALID_ARGUMENT;
    }
    const int64_t n = g->n_act;
    std::vector<float> planar((size_t)g->n_arrays * n);
    cpx_status s = cpx_grid_download_params(g, planar.data(), n);
    if (s != CPX_OK) return s;
    const int64_t WH = (int64_t)g->W * g->H;
    const int64_t cells = (int64_t)(g->W - 1) * (g->H - 1) * (g->D - 1);
    // occupancy.txt: the cell bytes of the last occupancy build (zeros before any)
    std::vector<uint8_t> occ((size_t)cells, 0);
    if (g->have_occupancy && g->occ_bytes)
        if (cudaMemcpy(occ.data(), g->occ_bytes, cells, cudaMemcpyDeviceToHost) != cudaSuccess)
            return cuda_status(cudaGetLastError(), "occupancy download");
    if (!write_ints(join(dir, "occupancy.txt"), occ.data(), g->D - 1, (int64_t)(g->W - 1) * (g->H - 1)))
        return io_error(join(dir, "occupancy.txt"), "writing");
    char name[256];
    if (!g->sparse) {
        std::snprintf(name, sizeof(name), "opacity_band%d.txt", band);
        if (!write_floats(join(dir, name), planar.data(), g->D, WH)) return io_error(join(dir, name), "writing");
    } else {
        std::snprintf(name, sizeof(name), "sparse_opacity_band%d.txt", band);
        if (!write_floats(join(dir, name), planar.data(), n, 1)) return io_error(join(dir, name), "writing");
        std::vector<uint32_t> idx((size_t)g->n_dense);
        if (cudaMemcpy(idx.data(), g->index_offsets, g->n_dense * 4, cudaMemcpyDeviceToHost) != cudaSuccess)
            return cuda_status(cudaGetLastError(), "sparse tables download");
        if (!write_ints(join(dir, "sparse_indexOffset.txt"), idx.data(), g->D, WH))
            return io_error(join(dir, "sparse_indexOffset.txt"), "writing");
        // the reference writes the in-cage flags to sparse_inCageInfo_band<b>.txt and then the
        // in-cage count over them (its fopen names inCageInfoFileName, SceneUtils.cu:1280-1283);
        // initFromFile reads the count from there.  The file that results holds the count alone.
        std::snprintf(name, sizeof(name), "sparse_inCageInfo_band%d.txt", band);
        FILE* f = std::fopen(join(dir, name).c_str(), "w");
        if (!f) return io_error(join(dir, name), "writing");
        std::fprintf(f, "%d", (int)g->in_cage_count);
        std::fclose(f);
    }
    if (density_only) return CPX_OK;
    const char* ch[3] = {"red", "green", "blue"};
    const int first = hierarchy_mode ? band * band : 0;
    for (int c = 0; c < 3; c++)
        for (int k = first; k < files_sh; k++) {
            const float* a = planar.data() + (size_t)(1 + c * g->sh_dim + k) * n;
            if (!g->sparse) {
                std::snprintf(name, sizeof(name), "%s_%d.txt", ch[c], k);
                if (!write_floats(join(dir, name), a, g->D, WH)) return io_error(join(dir, name), "writing");
            } else {
                std::snprintf(name, sizeof(name), "%s_%d_sparse.txt", ch[c], k);
                if (!write_floats(join(dir, name), a, n, 1)) return io_error(join(dir, name), "writing");
            }
        }
    return CPX_OK;
}

cpx_status cpx_grid_load_text(cpx_grid* g, const char* dir, int file_sh_dim)
{
    if (!g || !dir) {
        set_error("null argument");
        return CPX_ERR_INVALID_ARGUMENT;
    }
    if (g->sparse) {
        set_error("text checkpoints load into a dense grid");
        return CPX_ERR_UNSUPPORTED;
    }
    const int band = (int)(std::sqrt((double)file_sh_dim) - 1);
    if (file_sh_dim < 1 || (band + 1) * (band + 1) != file_sh_dim || file_sh_dim > g->sh_dim) {
        set_error("files of %d SH coefficients do not fit a grid of %d", file_sh_dim, g->sh_dim);
        return CPX_ERR_INVALID_ARGUMENT;
    }
    const int64_t n = g->n_act;
    std::vector<float> planar((size_t)g->n_arrays * n, 0.f);
    char name[256];
    std::snprintf(name, sizeof(name), "opacity_band%d.txt", band);
    if (!read_floats(join(dir, name), planar.data(), n)) return io_error(join(dir, name), "reading");
    const char* ch[3] = {"red", "green", "blue"};
    for (int c = 0; c < 3; c++)
        for (int k = 0; k < file_sh_dim; k++) {
            std::snprintf(name, sizeof(name), "%s_%d.txt", ch[c], k);
            if (!read_floats(join(dir, name), planar.data() + (size_t)(1 + c * g->sh_dim + k) * n, n))
                return io_error(join(dir, name), "reading");
        }
    return cpx_grid_upload_params(g, planar.data(), n);
}

cpx_status cpx_grid_download_occupancy(const cpx_grid* g, uint8_t* occupancy_out, uint8_t* in_cage_out,
                                       uint32_t* index_offsets_out, uint32_t* in_cage_count_out)
{
    if (!g) {
        set_error("null grid");
        return CPX_ERR_INVALID_ARGUMENT;
    }
    if (!g->have_occupancy) {
        set_error("the grid has no occupancy tables");
        return CPX_ERR_NOT_READY;
    }
    const int64_t C = (int64_t)(g->W - 1) * (g->H - 1) * (g->D - 1);
    cudaError_t e = cudaDeviceSynchronize();
    if (e == cudaSuccess && occupancy_out) e = cudaMemcpy(occupancy_out, g->occ_bytes, (size_t)C, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess && in_cage_out) e = cudaMemcpy(in_cage_out, g->in_cage, (size_t)g->n_dense, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess && index_offsets_out)
        e = cudaMemcpy(index_offsets_out, g->index_offsets, (size_t)g->n_dense * sizeof(uint32_t), cudaMemcpyDeviceToHost);
    if (in_cage_count_out) *in_cage_count_out = g->in_cage_count;
    return cuda_status(e, "download occupancy");
}

cpx_status cpx_grid_load_text_sparse(cpx_grid* g, const char* dir, int file_sh_dim)
{
    if (!g || !dir) {
        set_error("null argument");
        return CPX_ERR_INVALID_ARGUMENT;
    }
    if (g->sparse) {
        set_error("a sparse checkpoint loads into a fresh dense grid of its dimensions");
        return CPX_ERR_INVALID_ARGUMENT;
    }
    const int band = (int)(std::sqrt((double)file_sh_dim) - 1);
    if (file_sh_dim < 1 || (band + 1) * (band + 1) != file_sh_dim || file_sh_dim > g->sh_dim) {
        set_error("files of %d SH coefficients do not fit a grid of %d", file_sh_dim, g->sh_dim);
        return CPX_ERR_INVALID_ARGUMENT;
    }
    if (g->W < 2 || g->H < 2 || g->D < 2) {
        set_error("a sparse grid needs at least 2 vertices per axis");
        return CPX_ERR_INVALID_ARGUMENT;
    }
    char name[256];
    // the in-cage count, from the file initFromFile reads it from (SceneUtils.cu:725-733)
    std::snprintf(name, sizeof(name), "sparse_inCageInfo_band%d.txt", band);
    int count = -1;
    {
        FILE* f = std::fopen(join(dir, name).c_str(), "r");
        if (!f) return io_error(join(dir, name), "reading");
        const int got = std::fscanf(f, "%d", &count);
        std::fclose(f);
        if (got != 1 || count < 0 || count > g->n_dense) return io_error(join(dir, name), "reading the in-cage count of");
    }
    const int64_t N = g->n_dense;
    const int64_t C = (int64_t)(g->W - 1) * (g->H - 1) * (g->D - 1);
    std::vector<uint8_t> occ((size_t)C);
    if (!read_bytes(join(dir, "occupancy.txt"), occ.data(), C)) return io_error(join(dir, "occupancy.txt"), "reading");
    std::vector<uint32_t> idx((size_t)N);
    if (!read_u32(join(dir, "sparse_indexOffset.txt"), idx.data(), N))
        return io_error(join(dir, "sparse_indexOffset.txt"), "reading");
    const int64_t n = count;
    std::vector<float> planar((size_t)g->n_arrays * (n > 0 ? n : 1), 0.f);
    std::snprintf(name, sizeof(name), "sparse_opacity_band%d.txt", band);
    if (!read_floats(join(dir, name), planar.data(), n)) return io_error(join(dir, name), "reading");
    const char* ch[3] = {"red", "green", "blue"};
    for (int c = 0; c < 3; c++)
        for (int k = 0; k < file_sh_dim; k++) {
            std::snprintf(name, sizeof(name), "%s_%d_sparse.txt", ch[c], k);
            if (!read_floats(join(dir, name), planar.data() + (size_t)(1 + c * g->sh_dim + k) * n, n))
                return io_error(join(dir, name), "reading");
        }
    // occupancy tables from the saved cells: the in-cage flags by pruneScene's rule
    // (SceneUtils.cu:850-873), their prefix index, the brick map
    uint8_t* occ_dev = nullptr;
    cudaError_t e = cudaMalloc((void**)&occ_dev, (size_t)C);
    if (e == cudaSuccess) e = cudaMemcpy(occ_dev, occ.data(), (size_t)C, cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
        cudaFree(occ_dev);
        return cuda_status(e, "occupancy upload");
    }
    cpx_status rc = occupancy_build(g, 0.f, occ_dev);
    cudaFree(occ_dev);
    if (rc != CPX_OK) return rc;
    std::vector<uint32_t> built((size_t)N);
    e = cudaMemcpy(built.data(), g->index_offsets, (size_t)N * sizeof(uint32_t), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return cuda_status(e, "index offsets");
    if ((int64_t)g->in_cage_count != n || built != idx) {
        g->have_occupancy = 0;
        set_error("checkpoint %s is inconsistent: its occupancy gives %u in-cage vertices and %s index offsets, "
                  "the files say %d", dir, g->in_cage_count, built == idx ? "the same" : "other", count);
        return CPX_ERR_INVALID_ARGUMENT;
    }
    rc = make_sparse_launch(g);
    if (rc != CPX_OK) return rc;
    return cpx_grid_upload_params(g, planar.data(), n);
}

cpx_status cpx_image_load_text(const char* prefix, int width, int height, int gray_only, uint8_t* red, uint8_t* green,
                               uint8_t* blue, uint8_t* gray, uint8_t* mask, int* bbox)
{
    if (!prefix || width < 1 || height < 1 || !mask || !bbox || (gray_only ? !gray : (!red || !green || !blue))) {
        set_error("an image needs a prefix, its size and the planes to fill");
        return CPX_ERR_INVALID_ARGUMENT;
    }
    const int64_t n = (int64_t)width * height;
    const std::string p(prefix);
    // Image::initSelf's starting bounds (ImageUtils.cu:12-15), then readMask's, on the values
    // as read
    int b[4] = {height - 1, 0, width - 1, 0};
    FILE* mf = std::fopen((p + "_mask.txt").c_str(), "r");
    if (!mf) return io_error(p + "_mask.txt", "reading");
    for (int64_t i = 0; i < n; i++) {
        int v = 0;
        if (std::fscanf(mf, "%d ", &v) != 1) {
            std::fclose(mf);
            return io_error(p + "_mask.txt", "reading");
        }
        mask[i] = (uint8_t)v;
        if (!v) continue;
        const int row = (int)(i / width), col = (int)(i % width);
        if (row < b[0]) b[0] = row;
        if (row > b[1]) b[1] = row;
        if (col < b[2]) b[2] = col;
        if (col > b[3]) b[3] = col;
    }
    std::fclose(mf);
    for (int i = 0; i < 4; i++) bbox[i] = b[i];
    if (gray_only) return read_bytes(p + ".txt", gray, n) ? CPX_OK : io_error(p + ".txt", "reading");
    const char* suffix[3] = {"_red.txt", "_green.txt", "_blue.txt"};
    uint8_t* dst[3] = {red, green, blue};
    for (int c = 0; c < 3; c++)
        if (!read_bytes(p + suffix[c], dst[c], n)) return io_error(p + suffix[c], "reading");
    return CPX_OK;
}

cpx_status cpx_image_mask_pixels(const int* bbox, int width, int32_t* index_out, int64_t* n_out)
{
    if (!bbox || !n_out || width < 1) {
        set_error("null argument");
        return CPX_ERR_INVALID_ARGUMENT;
    }
    if (!(bbox[1] > bbox[0] && bbox[3] > bbox[2])) {  // processMasksInfo's assertion
        set_error("mask bounds [%d, %d] x [%d, %d] hold no rectangle", bbox[0], bbox[1], bbox[2], bbox[3]);
        return CPX_ERR_INVALID_ARGUMENT;
    }
    const int64_t n = (int64_t)(bbox[1] + 1 - bbox[0]) * (bbox[3] + 1 - bbox[2]);
    *n_out = n;
    if (!index_out) return CPX_OK;
    int64_t k = 0;
    for (int row = bbox[0]; row < bbox[1] + 1; row++)
        for (int col = bbox[2]; col < bbox[3] + 1; col++) index_out[k++] = row * width + col;
    return CPX_OK;
}

}  // extern "C"
