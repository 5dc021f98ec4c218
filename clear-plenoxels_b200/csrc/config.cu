// config.cu -- the reference's positional configuration file (readConfig, Utils.cu:765-932).
//
// The reference reads config.txt with one fscanf per line, in a fixed order ("SceneSize:%d %d
// %d\n", "RenderSize:%d %d\n", ...), so a file is valid only with every key present, in that
// order.  cpx_config_read parses the same lines with the same conversions into cpx_config.
// Unlike readConfig it checks each line (a missing or misordered key is an error naming it,
// where the reference would read on with the fields unset) and has no side effects: it creates
// no result directories, copies no files and does not seed the host's rand() -- the caller
// does what it needs of those (srand(random_seed) for the reference's jitter seeds).
#include <cstdio>
#include <cstring>

#include "cpx_internal.cuh"

using namespace cpx;

namespace {

struct Reader {
    FILE* f;
    const char* path;
    const char* failed = nullptr;
    // one line: `fmt` must convert `n` values
    template <typename... A>
    bool line(const char* key, const char* fmt, int n, A*... args)
    {
        if (failed) return false;
        if (std::fscanf(f, fmt, args...) != n) {
            failed = key;
            return false;
        }
        return true;
    }
};

}  // namespace

extern "C" cpx_status cpx_config_read(const char* path, cpx_config* out)
{
    if (!path || !out) {
        set_error("config: null argument");
        return CPX_ERR_INVALID_ARGUMENT;
    }
    FILE* f = std::fopen(path, "r");
    if (!f) {
        set_error("can not read config file: %s", path);
        return CPX_ERR_INVALID_ARGUMENT;
    }
    cpx_config c;
    std::memset(&c, 0, sizeof(c));
    c.huber_delta = 0.1f;  // Configuration's default (Utils.cuh)
    Reader r{f, path};
    // char arrays are read with %511s (the reference's %s into 512-byte fields)
    r.line("SceneSize", "SceneSize:%d %d %d\n", 3, &c.width, &c.height, &c.depth);
    r.line("RenderSize", "RenderSize:%d %d\n", 2, &c.render_width, &c.render_height);
    r.line("Graylized", "Graylized:%d\n", 1, &c.graylized);
    r.line("SphericalHarmonicsBand", "SphericalHarmonicsBand:%d\n", 1, &c.sh_band);
    r.line("HierarchyBandStrategy", "HierarchyBandStrategy:%d\n", 1, &c.hierarchy_band_strategy);
    r.line("SHsForTargetResolutionOnly", "SHsForTargetResolutionOnly:%d\n", 1, &c.shs_for_target_resolution_only);
    r.line("Hierarchy", "Hierarchy:%d\n", 1, &c.hierarchy);
    r.line("MinimumHierarchy", "MinimumHierarchy:%d\n", 1, &c.minimum_hierarchy);
    r.line("ToSparseHierarchy", "ToSparseHierarchy:%d\n", 1, &c.to_sparse_hierarchy);
    r.line("SilhouetteBound", "SilhouetteBound:%d\n", 1, &c.silhouette_bound);
    r.line("SilhouetteInitial", "SilhouetteInitial:%d\n", 1, &c.silhouette_initial);
    r.line("SilhouetteRadius", "SilhouetteRadius:%d\n", 1, &c.silhouette_radius);
    r.line("MaskAreaOnly", "MaskAreaOnly:%d\n", 1, &c.mask_area_only);
    r.line("InitialFromFile", "InitialFromFile:%d\n", 1, &c.initial_from_file);
    r.line("InitialFileDirBase", "InitialFileDirBase:%511s\n", 1, c.initial_file_dir_base);
    r.line("AvailableSHBands", "AvailableSHBands:%d\n", 1, &c.available_sh_bands);
    r.line("RenderOnly", "RenderOnly:%d\n", 1, &c.render_only);
    r.line("ViewDirectory", "ViewDirectory:%511s\n", 1, c.views_directory);
    r.line("CameraPoseFile", "CameraPoseFile:%511s\n", 1, c.camera_pose_file);
    r.line("ValidationPoseFile", "ValidationPoseFile:%511s\n", 1, c.validation_pose_file);
    r.line("NovelViewPoseFile", "NovelViewPoseFile:%511s\n", 1, c.novel_view_pose_file);
    r.line("CameraDistance", "CameraDistance:%lf\n", 1, &c.camera_distance);
    r.line("ViewCount", "ViewCount:%d\n", 1, &c.view_count);
    r.line("ValidationCount", "ValidationCount:%d\n", 1, &c.validation_count);
    r.line("TestCount", "TestCount:%d\n", 1, &c.test_count);
    r.line("TrainProcessViewIndex", "TrainProcessViewIndex:%d\n", 1, &c.train_process_view_index);
    r.line("WhiteBG", "WhiteBG:%d\n", 1, &c.white_bg);
    r.line("TestSkip", "TestSkip:%d\n", 1, &c.test_skip);
    r.line("RepeatLayers", "RepeatLayers:%d\n", 1, &c.repeat_layers);
    r.line("RandomSeed", "RandomSeed:%d\n", 1, &c.random_seed);
    r.line("LearningRate", "LearningRate:%lf\n", 1, &c.learning_rate);
    r.line("SHLearningRate", "SHLearningRate:%lf\n", 1, &c.sh_learning_rate);
    r.line("DensityOptimizer", "DensityOptimizer:%d\n", 1, &c.density_optimizer);
    r.line("ColorChannelOptimizer", "ColorChannelOptimizer:%d\n", 1, &c.color_channel_optimizer);
    r.line("Momentum", "Momentum:%lf\n", 1, &c.momentum);
    r.line("Epochs", "Epochs:%d\n", 1, &c.epochs);
    r.line("ValidationInterval", "ValidationInterval:%d\n", 1, &c.validation_interval);
    r.line("BatchSize", "BatchSize:%d\n", 1, &c.batch_size);
    r.line("FixBatchSize", "FixBatchSize:%d\n", 1, &c.fix_batch_size);
    r.line("BaseDir", "BaseDir:%511s\n", 1, c.base_dir);
    r.line("SaveIntervals", "SaveIntervals:%d\n", 1, &c.save_intervals);
    r.line("HalfLR", "HalfLR:%d\n", 1, &c.half_lr_intervals);
    r.line("LowestLR", "LowestLR:%lf\n", 1, &c.lowest_lr);
    r.line("PruneEpoch", "PruneEpoch:%d\n", 1, &c.prune_epoch);
    r.line("PruneThreshold", "PruneThreshold:%f\n", 1, &c.prune_threshold);
    r.line("Skips", "Skips:%d\n", 1, &c.skips);
    if (!r.failed && (c.skips < 0 || c.skips > CPX_CONFIG_MAX_SKIPS)) r.failed = "Skips (count out of range)";
    // "SkipIndex:%d " and then skips - 1 more "%d " (the first is read even with Skips:0)
    int first_skip = 0;
    r.line("SkipIndex", "SkipIndex:%d ", 1, &first_skip);
    if (!r.failed && c.skips > 0) c.skip_index[0] = first_skip;
    for (int i = 1; i < c.skips && !r.failed; i++) r.line("SkipIndex", "%d ", 1, &c.skip_index[i]);
    if (!r.failed) (void)!std::fscanf(f, "\n");
    r.line("StepSize", "StepSize:%f\n", 1, &c.step_size);
    r.line("SolidStrategy", "SolidStrategy:%d\n", 1, &c.solid_strategy);
    r.line("InitialDensity", "InitialDensity:%f\n", 1, &c.initial_density);
    r.line("InitialColor", "InitialColor:%f\n", 1, &c.initial_color);
    r.line("VarianceLossInterval", "VarianceLossInterval:%d\n", 1, &c.variance_loss_interval);
    r.line("VarianceCoefficient", "VarianceCoefficient:%lf\n", 1, &c.variance_coefficient);
    r.line("ColorDisparityCoefficient", "ColorDisparityCoefficient:%lf\n", 1, &c.sh_coefficient);
    r.line("MaskRayCoefficient", "MaskRayCoefficient:%lf\n", 1, &c.mask_ray_coefficient);
    r.line("VarianceType", "VarianceType:%d\n", 1, &c.variance_type);
    r.line("NeighboorNumsForTVLoss", "NeighboorNumsForTVLoss:%d\n", 1, &c.neighbour_nums);
    r.line("DiffuseRatio", "DiffuseRatio:%lf\n", 1, &c.diffuse_ratio);
    r.line("ExportModel", "ExportModel:%d\n", 1, &c.export_model);
    r.line("ShuffleRays", "ShuffleRays:%d\n", 1, &c.shuffle_rays);
    r.line("JustModel", "JustModel:%d\n", 1, &c.just_model);
    r.line("HuberDelta", "HuberDelta:%f\n", 1, &c.huber_delta);
    std::fclose(f);
    if (r.failed) {
        set_error("config %s: line %s missing or out of order", path, r.failed);
        return CPX_ERR_INVALID_ARGUMENT;
    }
    // the reference keeps these as bools: nonzero is true, except three that are true only at
    // 1 (Utils.cu:904-915)
    int* flags[] = {&c.graylized, &c.hierarchy_band_strategy, &c.shs_for_target_resolution_only,
                    &c.silhouette_bound, &c.silhouette_initial, &c.mask_area_only, &c.initial_from_file,
                    &c.render_only, &c.white_bg, &c.fix_batch_size, &c.solid_strategy};
    for (int* p : flags) *p = *p != 0;
    c.export_model = c.export_model == 1;
    c.shuffle_rays = c.shuffle_rays == 1;
    c.just_model = c.just_model == 1;
    *out = c;
    return CPX_OK;
}
