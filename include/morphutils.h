/*
 * morphutils.h -- drop-in declaration of the reference's getSdf, served by
 * libtaichi_b200.so (GPU thumbnail, morphology and contour tracing; no
 * OpenCV).
 *
 * Replaces the getSdf entry point and the Point_t struct of the reference's
 * morphutils.h (morphutils.h:24-27, 40-41) with the same C++ signature, so a
 * caller compiled against either header links against this library.  The
 * reference's other declarations there (Array2Mat, GetFileNamesInDir,
 * thinImage, imfill on cv::Mat, opencv_test, the timer macros) are OpenCV
 * helpers off the SpMV path and are not provided.
 */
#ifndef TAICHI_B200_MORPHUTILS_H
#define TAICHI_B200_MORPHUTILS_H

#include <string>
#include <vector>

#if defined(__GNUC__)
#define TAICHI_MORPH_API __attribute__((visibility("default")))
#else
#define TAICHI_MORPH_API
#endif

/* A thumbnail point: x = column, y = row (morphutils.h:24-27). */
struct Point_t {
    int x;
    int y;
};

/* Thumbnail shapes of a host CSR matrix (morohutils.cu:182-291): the
 * 512-row thumbnail, its morphology (hole fill, 30x1 and 1x30 openings,
 * subtraction, 5x5 diagonal opening) and its contours (RETR_CCOMP order, at
 * least 80 points).  Outputs as in the reference: category = "diagonal",
 * size = {512, thumbnail width}, shapeNum = number of contours kept,
 * shapePoints += {contour[0], contour[size/2]} per contour, widths +=
 * contourArea / |contour[0] - contour[size/2]| per contour.  A matrix of at
 * most 512 rows prints "the matrix is too small! exit" and returns with the
 * outputs untouched but category, as the reference does.  `path` is not read
 * (the reference uses only its file name, for nothing).  csrValHostPtr is not
 * read either.  Errors print "getSdf: <message>" and leave shapeNum = 0. */
TAICHI_MORPH_API void getSdf(std::string path, int M, int N, int nnz, int *&csrRowIndexHostPtr,
                             int *&csrColIndexHostPtr, float *&csrValHostPtr, std::string &category,
                             Point_t &size, int &shapeNum, std::vector<Point_t> &shapePoints,
                             std::vector<double> &widths);

#endif /* TAICHI_B200_MORPHUTILS_H */
