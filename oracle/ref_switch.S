/* Minimal x86-64 (System V) context switch for the host CUDA-block emulator
 * in oracle/ref_emu.cpp.  Test infrastructure only.
 *
 *   void lima_emu_switch(void** save_sp, void* to_sp);
 *
 * Saves the callee-saved registers, MXCSR and the x87 control word on the
 * current stack, stores the stack pointer in *save_sp, switches to to_sp and
 * restores the same set from there.  A fresh fiber stack is prepared by
 * prep_fiber_stack() in ref_emu.cpp with the identical frame layout.
 */
    .text
    .globl  lima_emu_switch
    .type   lima_emu_switch, @function
lima_emu_switch:
    pushq   %rbp
    pushq   %rbx
    pushq   %r12
    pushq   %r13
    pushq   %r14
    pushq   %r15
    subq    $8, %rsp
    stmxcsr (%rsp)
    fnstcw  4(%rsp)
    movq    %rsp, (%rdi)
    movq    %rsi, %rsp
    ldmxcsr (%rsp)
    fldcw   4(%rsp)
    addq    $8, %rsp
    popq    %r15
    popq    %r14
    popq    %r13
    popq    %r12
    popq    %rbx
    popq    %rbp
    ret
    .size   lima_emu_switch, .-lima_emu_switch
    .section .note.GNU-stack,"",@progbits
