/* Empty stand-in: the reference includes this MSVC/CUDA header but uses nothing from it on the host. */
#pragma once
