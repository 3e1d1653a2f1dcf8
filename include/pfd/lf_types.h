/*
 * lf_types.h -- the reference's matching-side data types, reduced to the
 * members the frame path reads and writes, for the C++ classes in this
 * directory (AdaptMIPMFrame.h, MIDisparityFilter.h, MICycleCheck.h).
 *
 * Each type keeps the reference's name, member names, member types and
 * ordering rules, so code written against the reference's
 *   MVStereo/LFDepthInfo.h  (PatchMatchParamsLF :19-46, MLA_Problem :175-268,
 *                            DisparityAndNormal :273-323)
 *   Common/Common.h         (LightFieldParams :155-185, LightFieldParamsCUDA :195-205)
 *   Common/CommonUtil.h     (MLA_Info :27-67)
 *   Common/QuadTree.h       (QuadTreeTileKey, operator< :137-148)
 * compiles against these.  Where the reference holds an OpenCV matrix
 * (cv::Mat, cv::Point2f), a plain stand-in with the same use is declared
 * here; a project that has the real headers includes those instead and
 * compiles the classes' .cpp files against them (the .cpp files use only the
 * members listed here).
 */
#ifndef PFD_LF_TYPES_H
#define PFD_LF_TYPES_H

#include <cstdint>
#include <map>
#include <memory>
#include <string>
#include <utility>
#include <vector>

#include <vector_types.h>   /* float2, float4, int2, int3 (CUDA's plain structs) */

namespace LFMVS {

/* cv::Point2f stand-in. */
struct Point2f {
    float x = 0.0f, y = 0.0f;
    Point2f() = default;
    Point2f(float x_, float y_) : x(x_), y(y_) {}
};

/* 8-bit single-channel cv::Mat stand-in (rows x cols, row-major, no padding).
 * The classes read images only through rows, cols, empty() and ptr(row), which
 * cv::Mat (CV_8UC1) has with the same meaning. */
struct GrayImage {
    int rows = 0, cols = 0;
    std::vector<uint8_t> data;
    GrayImage() = default;
    GrayImage(int r, int c, uint8_t fill = 0) : rows(r), cols(c), data((size_t)r * c, fill) {}
    bool empty() const { return rows <= 0 || cols <= 0 || data.empty(); }
    uint8_t* ptr(int row) { return data.data() + (size_t)row * cols; }
    const uint8_t* ptr(int row) const { return data.data() + (size_t)row * cols; }
};

/* Common/QuadTree.h: a tile (micro-image) key.  Maps order keys by
 * (LOD, row, column) through QuadTreeTileKeyMapCmpLess. */
class QuadTreeTileKey {
public:
    QuadTreeTileKey() = default;
    QuadTreeTileKey(int lod, int tile_x, int tile_y) : m_LOD(lod), m_TileX(tile_x), m_TileY(tile_y) {}
    int32_t GetLOD() const { return m_LOD; }
    int32_t GetTileX() const { return m_TileX; }   /* column */
    int32_t GetTileY() const { return m_TileY; }   /* row */
    bool operator==(const QuadTreeTileKey& r) const
    {
        return m_LOD == r.m_LOD && m_TileX == r.m_TileX && m_TileY == r.m_TileY;
    }
    bool operator<(const QuadTreeTileKey& r) const
    {
        if (m_LOD != r.m_LOD) return m_LOD < r.m_LOD;
        if (m_TileY != r.m_TileY) return m_TileY < r.m_TileY;
        return m_TileX < r.m_TileX;
    }

private:
    int32_t m_LOD = 0, m_TileX = 0, m_TileY = 0;
};
typedef std::shared_ptr<QuadTreeTileKey> QuadTreeTileKeyPtr;
typedef std::vector<QuadTreeTileKeyPtr> QuadTreeTileKeyPtrVec;

struct QuadTreeTileKeyMapCmpLess {
    bool operator()(const QuadTreeTileKeyPtr& a, const QuadTreeTileKeyPtr& b) const { return *a < *b; }
};

/* Common/CommonUtil.h:27-67: one lens of the calibrated micro-lens array. */
class MLA_Info {
public:
    void SetCenter(const Point2f& c) { m_Center = c; }
    Point2f& GetCenter() { return m_Center; }
    const Point2f& GetCenter() const { return m_Center; }
    void SetCol(int c) { m_Col = c; }
    int GetCol() const { return m_Col; }
    void SetRow(int r) { m_Row = r; }
    int GetRow() const { return m_Row; }
    void SetAbandonByArea(bool b) { m_BAbandon_area = b; }
    bool IsAbandonByArea() const { return m_BAbandon_area; }
    void SetArea(float a) { m_Area = a; }
    float& GetArea() { return m_Area; }

private:
    Point2f m_Center;
    int m_Col = 0, m_Row = 0;
    float m_Area = 0.0f;
    bool m_BAbandon_area = false;
};
typedef std::shared_ptr<MLA_Info> MLA_InfoPtr;
typedef std::map<QuadTreeTileKeyPtr, MLA_InfoPtr, QuadTreeTileKeyMapCmpLess> QuadTreeTileInfoMap;

/* Common/Common.h:155-185 (the members the matching path reads). */
struct LightFieldParams {
    int   mla_u_size = 0, mla_v_size = 0;
    int   mi_width_for_match = 0;
    int   mi_height_for_match = 0;
    float baseline = 0.0f;               /* lens pitch in pixels */
    float mainlen_flocal_length = 0.0f;
    float sensor_pixel_size = 0.0f;
};

/* Common/Common.h:195-205. */
struct LightFieldParamsCUDA {
    explicit LightFieldParamsCUDA(const LightFieldParams& p)
        : mi_width_for_match(p.mi_width_for_match), mia_height_for_match(p.mi_height_for_match), baseline(p.baseline)
    {
    }
    int   mi_width_for_match;
    int   mia_height_for_match;
    float baseline;
};

/* MVStereo/LFDepthInfo.h:19-46, same defaults. */
struct PatchMatchParamsLF {
    int   max_iterations = 3;
    int   patch_size = 5;
    int   patch_Bound_size = 5;
    int   propagation_Graph_size = 5;
    int   num_images = 18;
    int   max_image_size = 32000;
    int   radius_increment = 1;
    float sigma_spatial = 5.0f;
    float sigma_color = 3.0f;
    int   top_k = 5;
    float baseline = 0.54f;
    float depth_min = 5.0f;
    float depth_max = 40.0f;
    float disparity_min = 5.0f;
    float disparity_max = 40.0f;
    bool  geom_consistency = false;
    bool  multi_geometry = false;
    bool  planar_prior = false;
    float Base = 0;
    int   MLA_Mask_Width_Cuda = 0;
    int   MLA_Mask_Height_Cuda = 0;
    float base_height_ratio = 0.2f;
    float base_height_sigma = 0.05f;
    bool  b_test = false;
};

/* MVStereo/LFDepthInfo.h:114-140: a neighbour with its baseline (the fallback
 * neighbour list of the consistency pass when m_NeighsSortVecForMatch is empty). */
class Res_image_Key {
public:
    Res_image_Key(QuadTreeTileKeyPtr ptrKey, float baseline) : m_ptrKey(std::move(ptrKey)), Base_line(baseline) {}
    QuadTreeTileKeyPtr m_ptrKey;
    float Base_line = 0.0f;
};
typedef std::vector<Res_image_Key> Res_image_KeyVec;

/* MVStereo/LFDepthInfo.h:175-268: one micro-image's matching problem. */
class MLA_Problem {
public:
    bool                  m_bGarbage = false;     /* no depth wanted for this lens */
    bool                  m_bNeedMatch = true;
    QuadTreeTileKeyPtr    m_ptrKey;
    GrayImage             m_Image_gray;           /* mi_height x mi_width */
    GrayImage             m_Image_Blureness;      /* blur channel; empty = none */
    QuadTreeTileKeyPtrVec m_NeighsSortVecForMatch;/* neighbours, best first */
    Res_image_KeyVec      m_Res_Image_KeyVec;
};
typedef std::map<QuadTreeTileKeyPtr, MLA_Problem, QuadTreeTileKeyMapCmpLess> QuadTreeProblemMap;

/* Common/Common.h:142-152 (the frame path sets the first two). */
enum eStereoStage {
    eSS_ACMH_Begin = 0, eSS_ACMH_Finished, eSS_PlannerPrior_Begin, eSS_PlannerPrior_Finished,
    eSS_LRGeometric_Check, eSS_BlurFeature_Coarse, eSS_BlurFeature_Fine, eSS_BlurFeature_Finest
};

/* MVStereo/LFDepthInfo.h:273-323 and its constructor (LFDepthInfo.cpp:550-565):
 * per-micro-image result arrays of mi_width x mi_height, owned by new[]. */
class DisparityAndNormal {
public:
    explicit DisparityAndNormal(LightFieldParams& params);
    ~DisparityAndNormal();
    DisparityAndNormal(const DisparityAndNormal&) = delete;
    DisparityAndNormal& operator=(const DisparityAndNormal&) = delete;
    void Release();

    LightFieldParams   m_Params;
    QuadTreeTileKeyPtr m_ptrKey;
    float4*            ph_cuda = nullptr;        /* normal (x, y, z) + disparity (w) */
    float4*            disp_v_cuda = nullptr;    /* (d, d_real, |B|, |B| / d_real) */
    float*             c_cuda = nullptr;         /* matching cost */
    float*             d_cuda = nullptr;         /* disparity */
    unsigned int*      selected_views = nullptr; /* bit k: neighbour k selected */
    eStereoStage       m_StereoStage = eSS_ACMH_Begin;
    int                row = 0, col = 0;
};
typedef std::shared_ptr<DisparityAndNormal> DisparityAndNormalPtr;
typedef std::map<QuadTreeTileKeyPtr, DisparityAndNormalPtr, QuadTreeTileKeyMapCmpLess> QuadTreeDisNormalMap;

}  // namespace LFMVS

#endif
