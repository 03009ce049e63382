// tr_film_io.h - reference-compatible film output (host).
#pragma once
#include <cstdint>
#include <string>

namespace trio {

// Encodes one float RGB triple as Radiance RGBE (Ward, "Real Pixels", Graphics Gems II, 1991).
void rgbe_encode(float r, float g, float b, unsigned char out[4]);

// Writes a width x height float RGB image as an uncompressed Radiance .hdr file.
bool write_hdr(const std::string& path, uint32_t width, uint32_t height, const float* rgb, std::string* err);

// Writes what StreakCameraFilm::write produces (src/Film/StreakCameraFilm.h:233-242,356-437 and
// Film::average_and_write, src/Film/Film.h:357-471): for each scanline y an image
// "<name>_%04d.hdr" of width T (time) and height W (x), each row divided by that pixel's weight
// (NaN -> 0), transposed when T < 8; and the steady image "<name>.hdr" (W x H).  A null
// streak or steady skips that part.
bool write_streak_film(const char* name, uint32_t W, uint32_t H, uint32_t T, const double* streak,
                       const double* steady, const double* weight, std::string* err);

// Writes a film component averaged by the pixel weight (NaN -> 0) the way Film::average_and_write
// does (src/Film/Film.h:357-471, src/Image/ImageIO.h:146-193): ".hdr" as RGBE (one channel
// replicated to RGB, as stb's writer does), ".raw" as the float32 [H][W][channels] dump.
bool write_component(const std::string& path, uint32_t W, uint32_t H, uint32_t channels, const double* sums,
                     const double* weight, std::string* err);

}  // namespace trio
