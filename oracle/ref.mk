# Builds the reference library (tfhe v1.1, spqlios-fma FFT backend) straight from its
# own source files, without its CMake build system, into oracle/_ref/.
# The result is test infrastructure only: the parity checker and the timed CPU baseline.
#
#   make -f oracle/ref.mk REF=<reference checkout>       (run from the repository root)
#
# REF defaults to $TFHE_REFERENCE_DIR, else /root/reference.
#
# Flags follow the reference's "optim" build type (src/CMakeLists.txt:28: -O2 -DNDEBUG
# -funroll-loops), except that -march=native is replaced by -march=x86-64-v3 (AVX2+FMA, the
# ISA the spqlios-fma assembly needs) so the library also runs on other x86 hosts.
TFHE_REFERENCE_DIR ?= /root/reference
REF      ?= $(TFHE_REFERENCE_DIR)
SRC      := $(REF)/src/libtfhe
SPQ      := $(SRC)/fft_processors/spqlios
OUT      := oracle/_ref
OBJ      := $(OUT)/obj
CXX      ?= g++
CXXFLAGS := -std=gnu++11 -O2 -march=x86-64-v3 -DNDEBUG -funroll-loops -fPIC -w -I$(REF)/src/include

CORE := autogenerated lwebootstrappingkey lwe lwe-functions lwekey lwekeyswitch lweparams \
        lwesamples multiplication numeric-functions polynomials tgsw tlwe tlwe-functions \
        tgsw-functions tlwe-fft-operations tgsw-fft-operations toruspolynomial-functions \
        boot-gates lwe-keyswitch-functions lwe-bootstrapping-functions \
        lwe-bootstrapping-functions-fft tfhe_io tfhe_generic_streams tfhe_garbage_collector \
        tfhe_gate_bootstrapping tfhe_gate_bootstrapping_structures
FFTCPP := spqlios-fft-impl fft_processor_spqlios lagrangehalfc_impl
FFTASM := spqlios-fft-fma spqlios-ifft-fma lagrangehalfc_impl_fma

OBJS := $(addprefix $(OBJ)/core_,$(addsuffix .o,$(CORE))) \
        $(addprefix $(OBJ)/fft_,$(addsuffix .o,$(FFTCPP))) \
        $(addprefix $(OBJ)/asm_,$(addsuffix .o,$(FFTASM)))

all: $(OUT)/libtfhe-spqlios-fma.so $(OUT)/libtfhe_ref_shim.so

$(OBJ)/core_%.o: $(SRC)/%.cpp | $(OBJ)
	$(CXX) $(CXXFLAGS) -c $< -o $@
$(OBJ)/fft_%.o: $(SPQ)/%.cpp | $(OBJ)
	$(CXX) $(CXXFLAGS) -c $< -o $@
$(OBJ)/asm_%.o: $(SPQ)/%.s | $(OBJ)
	$(CXX) -c $< -o $@
$(OBJ):
	mkdir -p $@

$(OUT)/libtfhe-spqlios-fma.so: $(OBJS)
	$(CXX) -shared -Wl,-z,noexecstack -o $@ $^

# Thin extern "C" shim over the reference library: key generation, raw key export,
# gates, keyswitch and the multi-threaded CPU baseline, callable through ctypes.
$(OUT)/libtfhe_ref_shim.so: oracle/ref_shim.cpp $(OUT)/libtfhe-spqlios-fma.so
	$(CXX) $(CXXFLAGS) -shared -o $@ $< -L$(OUT) -ltfhe-spqlios-fma -Wl,-rpath,'$$ORIGIN' -lpthread

.PHONY: all
