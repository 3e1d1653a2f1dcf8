/*
 * pfd_calib.h -- the reference's on-disk calibration formats, read and written
 * on the host (part of libpfd.so; no device work).  Same conventions as
 * pfd_abi.h.
 *
 *  - intrinsics.xml: DepthSolver::ReadIntrinsicsFromXML (DepthSolver.cpp:872-1110),
 *    the camera model whose MLA pitch and grid size drive the matching window
 *    (mi = floor(pitch * 0.7071)) and the lens-centre detection;
 *  - CalibInfo.xml: DepthSolver::ReadCalibrationParamsFromXML (:1112-1250) and
 *    WriteCalibrationParamsXML (:1252-1340), the lens centres, keys, blur types
 *    and areas that the matcher's frame is built from (pfd_frame_create's
 *    centers and tilekeys).
 *
 * The readers take the text of the file (the caller reads it; nothing here
 * opens paths) and follow the reference's parse: the same elements, the same
 * sscanf conversions (%f to float, %lf to double, %d decimal, %i with C prefixes
 * for hex and octal), and the same quirks (the last "_" child of the pitch wins;
 * a later MLA with the same key replaces an earlier one; a lens type missing
 * from BlurInfo has blur radius 0).  Text the reference would crash on (an
 * element it dereferences missing, an element without text where it calls
 * GetText) gives PFD_EINVAL instead.
 */
#ifndef PFD_CALIB_H
#define PFD_CALIB_H

#include "pfd_abi.h"

#ifdef __cplusplus
extern "C" {
#endif

/* The LightFieldParams fields ReadIntrinsicsFromXML sets (Common/Common.h:155-205),
 * and the two globals it sets (D -> g_bl0, d -> g_B). */
typedef struct {
    float  D, d;                       /* root/D, root/d */
    double sensor_rotation[9];         /* row-major 3x3: sensor/pose/rotation, one "_" per column */
    double sensor_translate[3];        /* sensor/pose/translation/_ */
    float  sensor_pixel_size;          /* sensor/scale */
    float  mainlen_focal_length;       /* main_lens/f */
    int    mla_u_size, mla_v_size;     /* mia/mesh/width, height */
    float  baseline;                   /* mia/mesh/pitch/_/ : the last child */
    double distor_depth[3];            /* distortions/depth/_/ */
    double distor_radial[3];           /* distortions/radial/_/ */
    double distor_tangential[2];       /* distortions/tangential/_/ */
    int    has_mia;                    /* a mia group was present (bMIA) */
} pfd_intrinsics;

/* One micro-lens of CalibInfo.xml: MLA_Info's fields. */
typedef struct {
    int   col, row;                    /* key "row,col" */
    float cx, cy;                      /* center "x,y" */
    int   type;                        /* MLAType (eMLABlurType id), -1 when absent */
    float area;                        /* "aera" */
    float blur_radius;                 /* BlurInfo's radius of the type (0 when the type is not listed) */
} pfd_mla_entry;

/* Parses intrinsics.xml text (root "_"); fields the text does not set are 0. */
pfd_status pfd_read_intrinsics_xml(const char* text, pfd_intrinsics* out);

/* Parses CalibInfo.xml text (root "Calib").  The lenses come in the order of
 * the reference's m_MLA_info_map (key order: row, then column), duplicates
 * resolved as the map assignment does.  out may be NULL to count; *n receives
 * the number of lenses, and PFD_EINVAL is returned when it exceeds cap. */
pfd_status pfd_read_calib_xml(const char* text, pfd_mla_entry* out, int cap, int* n);

/* Writes CalibInfo.xml text as WriteCalibrationParamsXML does: BlurInfo with
 * types 0, 1, 2 (radius text = the id), then every lens in key order whose
 * abandon flag (may be NULL) is 0, with its key, centre, MLAType 1 and area,
 * numbers printed as a default std::ostream prints them (6 significant
 * digits), laid out as tinyxml2 prints a document (4-space indentation).
 * buf may be NULL to ask for the size; *len receives the text length without
 * the terminating NUL, and PFD_EINVAL is returned when buf_size <= *len. */
pfd_status pfd_write_calib_xml(const pfd_mla_entry* lenses, const int* abandon, int n, char* buf, size_t buf_size,
                               size_t* len);

#ifdef __cplusplus
}
#endif
#endif
