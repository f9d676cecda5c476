"""Drop-in modules for CLUEstering's Python wrapper (CLUEstering/CLUEstering.py).

The wrapper imports two nanobind extensions by name: CLUE_Convolutional_Kernels
(kernel classes and metric factories, CLUEstering/BindingModules/binding_kernels.cpp)
and one backend module per device type with listDevices() and mainRun()
(CLUEstering/BindingModules/Run.hpp:54-131). This directory holds pure-Python
modules with those names and signatures that call libclue_sm100.so through its
C ABI; put it on sys.path ahead of the wrapper's lib/ directory and the wrapper's
"gpu cuda" backend clusters on the B200.
"""
