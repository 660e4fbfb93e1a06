"""Python side of the B200 DSP-WENO stage path: ctypes binding of the C ABI
(include/dspw.h, libdspw.so) and the param.in helpers.  All compute runs in
libdspw.so; importing this package does not load CUDA."""
from .capi import (ABI_VERSION, BC, FLUX, MODEL, MU, PRECISION, RECON, TIME, Desc, DspwError,
                   Globals, Solver, StatusOut, TrainCfg, Trainer, check, lib, load_network_file, make_desc,
                   nvar, save_network_file, set_training_box, xavier_network)
from .paramfile import read_param, write_param
