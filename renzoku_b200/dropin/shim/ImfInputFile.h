/* Build stand-in for OpenEXR, which this image lacks (the reference's image I/O is never called here). */
#pragma once
