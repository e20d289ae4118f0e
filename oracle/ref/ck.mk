# TEST INFRASTRUCTURE ONLY -- included by oracle/Makefile once ref/ref_tree.py
# has prepared the reference tree in _ref/src.  Builds, from that tree:
#   _ref/adb_ref_ck_hash   hashing/ joins (PRO ... PMJ_*) with the checksum at the match sites
#   _ref/adb_ref_ck_sort   sorting/ joins (m-way, m-pass, m-way+skew) with the checksum
#   _ref/adb_ref_sort      sorting/ joins as the reference compiles them (the CPU baseline)
#   _ref/adb_ref_hash      hashing/ joins as the reference compiles them (the eager joins' CPU baseline)
#   _ref/adb_ref_hash_wait the same with WAIT kept, from _ref/src_wait (the eager joins' latency baseline)
TREE = _ref/src
CKFLAGS = -std=c++14 -O3 -pthread -msse4.2 -mavx2 -w -I ref/stub -I ref
HASH_SRC := $(wildcard $(TREE)/hashing/helper/*.cpp $(TREE)/hashing/joins/*.cpp $(TREE)/hashing/timer/*.cpp \
                       $(TREE)/hashing/utils/*.cpp)
HASH_SRC := $(filter-out %/fetcher_old.cpp,$(HASH_SRC))
SORT_SRC := $(wildcard $(TREE)/sorting/affinity/*.cpp $(TREE)/sorting/datagen/*.cpp $(TREE)/sorting/joins/*.cpp \
                       $(TREE)/sorting/timer/*.cpp $(TREE)/sorting/utils/*.cpp)
HASH_CK_OBJ := $(patsubst $(TREE)/%.cpp,_ref/obj_ck/%.o,$(HASH_SRC))
SORT_CK_OBJ := $(patsubst $(TREE)/%.cpp,_ref/obj_ck/%.o,$(SORT_SRC))
SORT_OBJ := $(patsubst $(TREE)/%.cpp,_ref/obj/%.o,$(SORT_SRC))
HASH_OBJ := $(patsubst $(TREE)/%.cpp,_ref/obj/%.o,$(HASH_SRC))

ck-all: _ref/adb_ref_ck_hash _ref/adb_ref_ck_sort _ref/adb_ref_sort _ref/adb_ref_hash

# the hashing/ joins with the reference's WAIT kept (tree _ref/src_wait):
# tuples released at their arrival times, the eager joins' latency baseline
TREE_W = _ref/src_wait
HASH_W_SRC := $(wildcard $(TREE_W)/hashing/helper/*.cpp $(TREE_W)/hashing/joins/*.cpp $(TREE_W)/hashing/timer/*.cpp \
                         $(TREE_W)/hashing/utils/*.cpp)
HASH_W_SRC := $(filter-out %/fetcher_old.cpp,$(HASH_W_SRC))
HASH_W_OBJ := $(patsubst $(TREE_W)/%.cpp,_ref/obj_wait/%.o,$(HASH_W_SRC))

wait-all: _ref/adb_ref_hash_wait

_ref/obj_wait/hashing/%.o: $(TREE_W)/hashing/%.cpp ref/checksum.h
	@mkdir -p $(dir $@)
	$(CXX) $(CKFLAGS) -DADB_REF_NO_CK -I $(TREE_W)/hashing -include ref/checksum.h -c $< -o $@

_ref/obj_wait/harness_hash.o: ref/harness.cpp ref/gen.h ref/checksum.h
	@mkdir -p $(dir $@)
	$(CXX) $(CKFLAGS) -DADB_REF_FULL -DADB_REF_NO_CK -I $(TREE_W)/hashing -include ref/checksum.h -c $< -o $@

_ref/adb_ref_hash_wait: $(HASH_W_OBJ) _ref/obj_wait/harness_hash.o
	$(CXX) -pthread -o $@ $^

_ref/obj_ck/hashing/%.o: $(TREE)/hashing/%.cpp ref/checksum.h
	@mkdir -p $(dir $@)
	$(CXX) $(CKFLAGS) -I $(TREE)/hashing -include ref/checksum.h -c $< -o $@

_ref/obj_ck/sorting/%.o: $(TREE)/sorting/%.cpp ref/checksum.h
	@mkdir -p $(dir $@)
	$(CXX) $(CKFLAGS) -I $(TREE)/sorting -include ref/checksum.h -c $< -o $@

_ref/obj/hashing/%.o: $(TREE)/hashing/%.cpp ref/checksum.h
	@mkdir -p $(dir $@)
	$(CXX) $(CKFLAGS) -DADB_REF_NO_CK -I $(TREE)/hashing -include ref/checksum.h -c $< -o $@

_ref/obj/harness_hash.o: ref/harness.cpp ref/gen.h ref/checksum.h
	@mkdir -p $(dir $@)
	$(CXX) $(CKFLAGS) -DADB_REF_FULL -DADB_REF_NO_CK -I $(TREE)/hashing -include ref/checksum.h -c $< -o $@

_ref/adb_ref_hash: $(HASH_OBJ) _ref/obj/harness_hash.o
	$(CXX) -pthread -o $@ $^

_ref/obj/sorting/%.o: $(TREE)/sorting/%.cpp ref/checksum.h
	@mkdir -p $(dir $@)
	$(CXX) $(CKFLAGS) -DADB_REF_NO_CK -I $(TREE)/sorting -include ref/checksum.h -c $< -o $@

_ref/obj_ck/harness_hash.o: ref/harness.cpp ref/gen.h ref/checksum.h
	@mkdir -p $(dir $@)
	$(CXX) $(CKFLAGS) -DADB_REF_CK -I $(TREE)/hashing -include ref/checksum.h -c $< -o $@

_ref/obj_ck/harness_sort.o: ref/harness_sort.cpp ref/gen.h ref/checksum.h
	@mkdir -p $(dir $@)
	$(CXX) $(CKFLAGS) -DADB_REF_CK -I $(TREE)/sorting -include ref/checksum.h -c $< -o $@

_ref/obj/harness_sort.o: ref/harness_sort.cpp ref/gen.h ref/checksum.h
	@mkdir -p $(dir $@)
	$(CXX) $(CKFLAGS) -DADB_REF_NO_CK -I $(TREE)/sorting -include ref/checksum.h -c $< -o $@

_ref/adb_ref_ck_hash: $(HASH_CK_OBJ) _ref/obj_ck/harness_hash.o
	$(CXX) -pthread -o $@ $^

_ref/adb_ref_ck_sort: $(SORT_CK_OBJ) _ref/obj_ck/harness_sort.o
	$(CXX) -pthread -o $@ $^

_ref/adb_ref_sort: $(SORT_OBJ) _ref/obj/harness_sort.o
	$(CXX) -pthread -o $@ $^

.PHONY: ck-all wait-all
