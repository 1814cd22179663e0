/* The reference's src/image_util.c:3406 calls sp_image_write (src/image_io.c:
 * HDF5/TIFF/PNG writers), which is not on the phasing path and whose libraries
 * are absent.  The oracle build links this stand-in, which writes nothing. */
#include <stdio.h>
typedef struct Image Image;
void sp_image_write(const Image *img, const char *filename, long long flags) {
  (void)img; (void)flags;
  fprintf(stderr, "oracle build: sp_image_write(%s) is not available\n", filename);
}
