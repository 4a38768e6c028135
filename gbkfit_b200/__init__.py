"""B200-native GBKFIT model-evaluation path (smdisk/mcdisk -> PSF x LSF FFT
convolution -> moments -> chi^2) behind the reference driver API."""
